// CPU FP64 oracle for the LBM_Mutiwing time step — TEST INFRASTRUCTURE ONLY.
//
// A sequential restatement of the reference Fortran solver's CPU semantics
// (OpenACC directives ignored, numprocs=1, max_meshid=1, bc_num=4), written
// so that the order of floating-point operations follows the Fortran source
// expression by expression.  It is compiled with -ffp-contract=off so that no
// multiply-add is fused.  Only tests/, the smoke check and the benchmark's
// CPU-baseline leg load it; the product library never links or calls it.
//
// Parity status: "parity unpinned" against the reference binary (no Fortran
// compiler exists here and the reference ships no golden vectors).  The
// restatement is pinned by the known-answer tests in tests/test_oracle_kat.py.
//
// Citations are file:line in the reference project (R-IFFERY/LBM_Mutiwing).
// Two documented deviations, both without effect on results:
//  * init's first move_boundary (solution.f90:74) runs before read_boundary
//    with zero geometry; the band it builds is cleared at step 1 and every
//    field it touches is already zero, so the oracle starts with an empty band.
//  * boundary_condition1's corner precompute (boundary_condition.f90:302-401)
//    and the first top/bottom LODI loops (:585-625, :713-755) are overwritten
//    before use (:655-661, :782-788) and are not evaluated.
// Deliberate generalisations: wings may have different marker counts, and
// wing_count = 0 (no immersed body) is accepted for uniform-flow tests.

#include "lbm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <thread>

namespace {

const double PAI = 3.1415926535897932384626433832795;  // main.f90:9

struct Ora {
    OraConfig c{};
    int Nx = 0, Ny = 0, N = 0;
    double niu = 0, tau = 0, UU = 0, scale = 0, ox = 0, oy = 0;
    double s[10]{};
    int e[10][3]{};
    double w[10]{};
    double matm[10][10]{}, minv[10][10]{};
    std::vector<double> f, f0, rho, u, v, u0, v0, pre, gfx, gfy;
    std::vector<int> body, bandidx;
    // geometry (airfoil.f90:207-242)
    int W = 0, npts = 0, nseg = 0;
    std::vector<int> pts, pstart, sstart, seg_wing;
    std::vector<double> xb0, yb0, xb1, yb1, xb2, yb2, arc;
    // band (airfoil.f90:286-335)
    std::vector<int> ap_i, ap_j, ap_w;
    // motion state (main.f90:72-80)
    std::vector<double> angle, omega, omgac, sa, sau, saac, sb, sbv, sbac;
    std::vector<double> rel_v, rel_s, rel_pos, extra_v, extra_s, extra_pos;
    int movenum = 0;
    int ncol = 0;
    std::vector<double> table;   // nrows x ncol
    int64_t table_rows = 0;
    std::vector<double> step_table;
    int64_t step_rows = 0;
    double motion_dt = 0, motion_end_time = 0;
    int64_t motion_index = 1;
    std::vector<double> stream_start, stream_target;
    bool stream_ready = false;
    double time = 0, err = 0;
    std::vector<double> wing_force, wing_moment;  // W*2, W
    std::vector<double> sum_row;
    int sample_count = 0, row_len = 0;
    double ibm_resid = 0;
    int nthreads = 1;

    size_t IX(int i, int j) const { return (size_t)(j - 1) * Nx + (i - 1); }
    double& F(int i, int j, int k) { return f[(size_t)(k - 1) * N + IX(i, j)]; }
    double& F0(int i, int j, int k) { return f0[(size_t)(k - 1) * N + IX(i, j)]; }
};

// Runs body(j) for j in [lo, hi] on nthreads threads, contiguous row blocks.
// Each row is computed independently, so results do not depend on nthreads.
template <class Fn>
void par_rows(int nthreads, int lo, int hi, Fn body) {
    int n = hi - lo + 1;
    if (nthreads <= 1 || n < 64) {
        for (int j = lo; j <= hi; ++j) body(j);
        return;
    }
    std::vector<std::thread> th;
    int per = (n + nthreads - 1) / nthreads;
    for (int t = 0; t < nthreads; ++t) {
        int a = lo + t * per, b = std::min(hi, a + per - 1);
        if (a > b) break;
        th.emplace_back([=]() { for (int j = a; j <= b; ++j) body(j); });
    }
    for (auto& x : th) x.join();
}

// matmulvoc (boundary_condition.f90:1738-1755): c(i) = sum_j a(i,j) b(j)
inline void matmulvoc(double* c, const double a[10][10], const double* b) {
    for (int i = 1; i <= 9; ++i) {
        double sum = 0.0;
        for (int j = 1; j <= 9; ++j) sum = sum + a[i][j] * b[j];
        c[i] = sum;
    }
}

// nizhen (solution.f90:1474-1529): Gauss-Jordan inverse with partial
// pivoting, including its in-loop pivot-row normalisation.
void nizhen(const double AA[10][10], double b1[10][10], int Nm) {
    double a[10][10];
    for (int i = 1; i <= Nm; ++i)
        for (int j = 1; j <= Nm; ++j) { a[i][j] = AA[i][j]; b1[i][j] = 0.0; }
    for (int k = 1; k <= Nm; ++k) b1[k][k] = 1.0;
    double temp, mik;
    for (int k = 1; k <= Nm - 1; ++k) {
        int ik = k;
        temp = std::fabs(a[ik][k]);
        for (int i = k; i <= Nm; ++i)
            if (std::fabs(a[i][k]) > std::fabs(temp)) { temp = std::fabs(a[i][k]); ik = i; }
        for (int j = 1; j <= Nm; ++j) {
            temp = a[ik][j]; a[ik][j] = a[k][j]; a[k][j] = temp;
            temp = b1[ik][j]; b1[ik][j] = b1[k][j]; b1[k][j] = temp;
        }
        for (int i = 1; i <= Nm; ++i) {
            mik = a[i][k] / a[k][k];
            temp = a[k][k];
            for (int j = k; j <= Nm; ++j)
                if (i != k) a[i][j] = a[i][j] - mik * a[k][j];
            for (int j = k; j <= Nm; ++j) a[k][j] = a[k][j] / temp;
            for (int j = 1; j <= Nm; ++j)
                if (i != k) b1[i][j] = b1[i][j] - mik * b1[k][j];
            for (int j = 1; j <= Nm; ++j) b1[k][j] = b1[k][j] / temp;
        }
    }
    temp = a[Nm][Nm];
    for (int i = 1; i <= Nm - 1; ++i) {
        mik = a[i][Nm] / a[Nm][Nm];
        a[i][Nm] = 0.0;
        for (int j = 1; j <= Nm; ++j) b1[i][j] = b1[i][j] - mik * b1[Nm][j];
    }
    a[Nm][Nm] = 1.0;
    for (int j = 1; j <= Nm; ++j) b1[Nm][j] = b1[Nm][j] / temp;
}

void set_matm(Ora& o) {
    // solution.f90:17-25
    static const double M[9][9] = {
        {1, 1, 1, 1, 1, 1, 1, 1, 1},   {-4, -1, -1, -1, -1, 2, 2, 2, 2},
        {4, -2, -2, -2, -2, 1, 1, 1, 1}, {0, 1, 0, -1, 0, 1, -1, -1, 1},
        {0, -2, 0, 2, 0, 1, -1, -1, 1}, {0, 0, 1, 0, -1, 1, 1, -1, -1},
        {0, 0, -2, 0, 2, 1, 1, -1, -1}, {0, 1, -1, 1, -1, 0, 0, 0, 0},
        {0, 0, 0, 0, 0, 1, -1, 1, -1}};
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) o.matm[i + 1][j + 1] = M[i][j];
    nizhen(o.matm, o.minv, 9);
}

void d2q9model(Ora& o) {
    // D2Q9model.f90:5-32; weights are single-precision literals stored in FP64.
    static const int ex[9] = {0, 1, 0, -1, 0, 1, -1, -1, 1};
    static const int ey[9] = {0, 0, 1, 0, -1, 1, 1, -1, -1};
    for (int k = 1; k <= 9; ++k) { o.e[k][1] = ex[k - 1]; o.e[k][2] = ey[k - 1]; }
    o.w[1] = (double)(4.0f / 9.0f);
    for (int k = 2; k <= 5; ++k) o.w[k] = (double)(1.0f / 9.0f);
    for (int k = 6; k <= 9; ++k) o.w[k] = (double)(1.0f / 36.0f);
}

// D2Q9feq (D2Q9model.f90:35-46)
inline double d2q9feq(const Ora& o, double rh, double u1, double v1, int k) {
    double eu = (double)o.e[k][1] * u1 + (double)o.e[k][2] * v1;
    double utwo = u1 * u1 + v1 * v1;
    return o.w[k] * rh * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * utwo);
}

// ---------------------------------------------------------------- motion
// apply_motion_row (mode.f90:180-218)
void apply_motion_row(Ora& o, const double* row) {
    for (int w = 0; w < o.W; ++w) {
        int col = 1 + w * 9;  // 0-based index of the wing's first column
        o.angle[w] = row[col]; o.omega[w] = row[col + 1]; o.omgac[w] = row[col + 2];
        o.sa[w] = row[col + 3]; o.sau[w] = row[col + 4]; o.saac[w] = row[col + 5];
        o.sb[w] = row[col + 6]; o.sbv[w] = row[col + 7]; o.sbac[w] = row[col + 8];
        if (o.c.motion_source == 1) {
            double x_base = o.c.wing_x_origin + (double)w * o.c.wing_x_spacing;
            double y_base = o.c.wing_y_origin;
            o.sa[w] = o.sa[w] - x_base;
            o.sb[w] = o.sb[w] - y_base;
        }
    }
}

// smooth_r/h/d (mode.f90:220-261)
double smooth_r(double x) {
    if (x < 0.0) return 0.0;
    if (x <= 1.0) return 0.5 * x * x + (std::cos(2.0 * PAI * x) - 1.0) / (4.0 * PAI * PAI);
    return x - 0.5;
}
double smooth_h(double x) {
    if (x < 0.0) return 0.0;
    if (x <= 1.0) return x - std::sin(2.0 * PAI * x) / (2.0 * PAI);
    return 1.0;
}
double smooth_d(double x) {
    if (x >= 0.0 && x <= 1.0) return 1.0 - std::cos(2.0 * PAI * x);
    return 0.0;
}

// interpolate_motion_triplet (mode.f90:263-285)
void triplet(double s0, double v0, double v1, double dt, double local_t, double* s, double* v,
             double* a) {
    double delta_v = v1 - v0;
    if (dt <= 1.0e-14) {
        *s = (v0 + delta_v) * local_t + s0;
        *v = v0 + delta_v;
        *a = 0.0;
        return;
    }
    double x = local_t / dt;
    *s = delta_v * dt * smooth_r(x) + v0 * local_t + s0;
    *v = delta_v * smooth_h(x) + v0;
    *a = delta_v / dt * smooth_d(x);
}

// interpolate_motion_row / lookup_motion_row (mode.f90:327-386)
void interpolate_motion_row(Ora& o, int64_t i1, int64_t i2, double target, double* row) {
    const double* r1 = &o.table[(size_t)(i1 - 1) * o.ncol];
    const double* r2 = &o.table[(size_t)(i2 - 1) * o.ncol];
    double t1 = r1[0], t2 = r2[0], dt = t2 - t1;
    if (std::fabs(dt) <= 1.0e-14) {
        for (int c = 0; c < o.ncol; ++c) row[c] = r2[c];
        row[0] = target;
        return;
    }
    double ratio = (target - t1) / dt;
    ratio = std::min(std::max(ratio, 0.0), 1.0);
    for (int c = 0; c < o.ncol; ++c) row[c] = r1[c] + ratio * (r2[c] - r1[c]);
    row[0] = target;
}

void lookup_motion_row(Ora& o, double target, double* row) {
    const double tol = 1.0e-12;
    int64_t np = o.table_rows;
    if (target <= o.table[0] + tol) {
        o.motion_index = 1;
        for (int c = 0; c < o.ncol; ++c) row[c] = o.table[c];
        row[0] = target;
        return;
    }
    if (target >= o.table[(size_t)(np - 1) * o.ncol] - tol) {
        o.motion_index = np;
        for (int c = 0; c < o.ncol; ++c) row[c] = o.table[(size_t)(np - 1) * o.ncol + c];
        row[0] = target;
        return;
    }
    o.motion_index = std::max<int64_t>(1, std::min<int64_t>(o.motion_index, np - 1));
    while (o.motion_index > 1 && target <= o.table[(size_t)(o.motion_index - 1) * o.ncol] + tol)
        o.motion_index -= 1;
    while (o.motion_index < np - 1 && target > o.table[(size_t)(o.motion_index) * o.ncol] + tol)
        o.motion_index += 1;
    interpolate_motion_row(o, o.motion_index, o.motion_index + 1, target, row);
}

// lookup_stream_motion_row (mode.f90:414-449)
void lookup_stream_row(Ora& o, double target, double* row) {
    const double tol = 1.0e-12;
    double t1 = o.stream_start[0], t2 = o.stream_target[0], dt = t2 - t1;
    if (target <= t1 + tol) {
        for (int c = 0; c < o.ncol; ++c) row[c] = o.stream_start[c];
        row[0] = target;
        return;
    }
    double local_t = std::min(std::max(target - t1, 0.0), std::max(dt, 0.0));
    for (int c = 0; c < o.ncol; ++c) row[c] = 0.0;
    row[0] = target;
    for (int w = 0; w < o.W; ++w) {
        int col = 1 + w * 9;
        for (int t = 0; t < 3; ++t) {
            int cc = col + 3 * t;
            triplet(o.stream_start[cc], o.stream_start[cc + 1], o.stream_target[cc + 1], dt, local_t,
                    &row[cc], &row[cc + 1], &row[cc + 2]);
        }
    }
}

// mode (mode.f90:451-471)
int mode(Ora& o) {
    if (o.W == 0) return 0;   // no immersed body, nothing to move
    std::vector<double> row(o.ncol);
    if (o.c.motion_source == 2) {
        if (!o.stream_ready) return -1;
        lookup_stream_row(o, o.time, row.data());
        apply_motion_row(o, row.data());
        return 0;
    }
    if (o.step_rows <= 0 || o.motion_dt <= 0.0) return -1;
    int64_t idx = (int64_t)std::llround(o.time / o.motion_dt) + 1;
    idx = std::max<int64_t>(1, std::min<int64_t>(idx, o.step_rows));
    apply_motion_row(o, &o.step_table[(size_t)(idx - 1) * o.ncol]);
    return 0;
}

// update_body_extra_from_rel (mode.f90:473-495)
void update_body_extra(Ora& o) {
    double av = 0, as = 0, ap = 0;
    for (int w = 0; w < o.W; ++w) {
        av = av + o.rel_v[w]; as = as + o.rel_s[w]; ap = ap + o.rel_pos[w];
        o.extra_v[w] = av; o.extra_s[w] = as; o.extra_pos[w] = ap;
    }
}

// ---------------------------------------------------------------- geometry
// move_boundary (airfoil.f90:244-338)
void move_boundary(Ora& o) {
    for (int w = 0; w < o.W; ++w) {
        int ps = o.pstart[w], ss = o.sstart[w];
        double ca = std::cos(o.angle[w]), sn = std::sin(o.angle[w]);
        for (int p = ps; p < ps + o.pts[w]; ++p) {
            o.xb1[p] = ca * o.xb0[p] + sn * o.yb0[p] + o.c.wing_x_origin +
                       (double)w * o.c.wing_x_spacing + o.sa[w] + o.c.xc +
                       o.extra_s[w] / (1.0 / o.scale) - (double)o.movenum * o.scale;
            o.yb1[p] = -(sn * o.xb0[p]) + ca * o.yb0[p] + o.c.wing_y_origin + o.sb[w] + o.c.yc;
        }
        for (int sg = ss; sg < ss + o.pts[w] - 1; ++sg) {
            int p = ps + (sg - ss);
            o.xb2[sg] = 0.5 * (o.xb1[p + 1] + o.xb1[p]);
            o.yb2[sg] = 0.5 * (o.yb1[p + 1] + o.yb1[p]);
        }
    }
    for (size_t b = 0; b < o.ap_i.size(); ++b) {
        size_t id = o.IX(o.ap_i[b], o.ap_j[b]);
        o.body[id] = 0;
        o.gfx[id] = 0.0;
        o.gfy[id] = 0.0;
        o.bandidx[id] = -1;
    }
    o.ap_i.clear(); o.ap_j.clear(); o.ap_w.clear();
    for (int sg = 0; sg < o.nseg; ++sg) {
        int wing = o.seg_wing[sg];
        double x2 = o.xb2[sg], y2 = o.yb2[sg];
        int i1 = (int)((x2 - o.ox) / o.scale + 1.0);
        for (int i = i1; i >= 1; --i) {
            double t = o.ox + (double)(i - 1) * o.scale;
            if (std::fabs((t - x2) / o.scale) > 2.5) { i1 = i + 1; break; }
        }
        int i2 = (int)((x2 - o.ox) / o.scale + 1.0);
        for (int i = i2; i <= o.Nx; ++i) {
            double t = o.ox + (double)(i - 1) * o.scale;
            if (std::fabs((t - x2) / o.scale) > 2.5) { i2 = i - 1; break; }
        }
        int j2 = (int)((y2 - o.oy) / o.scale + 1.0);
        for (int i = j2; i <= o.Ny; ++i) {
            double t = o.oy + (double)(i - 1) * o.scale;
            if (std::fabs((t - y2) / o.scale) > 2.5) { j2 = i - 1; break; }
        }
        int j1 = (int)((y2 - o.oy) / o.scale + 1.0);
        for (int i = j1; i >= 1; --i) {
            double t = o.oy + (double)(i - 1) * o.scale;
            if (std::fabs((t - y2) / o.scale) > 2.5) { j1 = i + 1; break; }
        }
        for (int i = i1; i <= i2; ++i)
            for (int j = j1; j <= j2; ++j) {
                size_t id = o.IX(i, j);
                if (o.body[id] == 0) {
                    o.body[id] = 1;
                    o.bandidx[id] = (int)o.ap_i.size();
                    o.ap_i.push_back(i); o.ap_j.push_back(j); o.ap_w.push_back(wing);
                }
            }
    }
}

// ---------------------------------------------------------------- lattice
// streaming (solution.f90:440-481)
void streaming(Ora& o) {
    par_rows(o.nthreads, 2, o.Ny - 1, [&](int j) {
        for (int k = 1; k <= 9; ++k)
            for (int i = 2; i <= o.Nx - 1; ++i)
                o.F0(i, j, k) = o.F(i - o.e[k][1], j - o.e[k][2], k);
    });
}

// physical_variables (solution.f90:483-583)
void physical_variables(Ora& o) {
    par_rows(o.nthreads, 1, o.Ny, [&](int j) {
        for (int i = 1; i <= o.Nx; ++i) {
            size_t id = o.IX(i, j);
            o.u0[id] = o.u[id];
            o.v0[id] = o.v[id];
            double trho = 0.0, tu = 0.0, tv = 0.0;
            bool border = (i == 1) || (i == o.Nx) || (j == 1) || (j == o.Ny);
            for (int k = 1; k <= 9; ++k) {
                double t = o.F0(i, j, k);
                if (!border) o.F(i, j, k) = t;
                trho = trho + t;
                tu = tu + (double)o.e[k][1] * t;
                tv = tv + (double)o.e[k][2] * t;
            }
            o.rho[id] = trho;
            o.pre[id] = trho / 3.0;
            o.u[id] = tu / trho;
            o.v[id] = tv / trho;
        }
    });
}

// colission (solution.f90:585-669)
void colission(Ora& o) {
    const double* s = o.s;
    par_rows(o.nthreads, 2, o.Ny - 1, [&](int j) {
        for (int i = 2; i <= o.Nx - 1; ++i) {
            double temp[10], temp1[10], fp[10];
            for (int k = 1; k <= 9; ++k) temp[k] = o.F(i, j, k);
            matmulvoc(temp1, o.matm, temp);
            size_t id = o.IX(i, j);
            double ut = o.u[id], vt = o.v[id], rt = o.rho[id];
            temp[1] = 0.0;
            temp[2] = -2.0 * rt + 3.0 * (rt * ut * rt * ut + rt * vt * rt * vt);
            temp[3] = rt - 3.0 * (rt * ut * rt * ut + rt * vt * rt * vt);
            temp[4] = 0.0;
            temp[5] = -(rt * ut);
            temp[6] = 0.0;
            temp[7] = -(rt * vt);
            temp[8] = (rt * ut * rt * ut - rt * vt * rt * vt);
            temp[9] = (rt * ut * rt * vt);
            double gx = o.gfx[id], gy = o.gfy[id];
            fp[1] = 0.0;
            fp[2] = 6.0 * (1.0 - 0.5 * s[2]) * (ut * gx + vt * gy);
            fp[3] = -(6.0 * (1.0 - 0.5 * s[3]) * (ut * gx + vt * gy));
            fp[4] = gx;
            fp[5] = -((1.0 - 0.5 * s[5]) * gx);
            fp[6] = gy;
            fp[7] = -((1.0 - 0.5 * s[7]) * gy);
            fp[8] = 2.0 * (1.0 - 0.5 * s[8]) * (ut * gx - vt * gy);
            fp[9] = (1.0 - 0.5 * s[9]) * (ut * gy + vt * gx);
            for (int k = 1; k <= 9; ++k) temp[k] = temp1[k] + (temp[k] - temp1[k]) * s[k] + fp[k];
            matmulvoc(temp1, o.minv, temp);
            for (int k = 1; k <= 9; ++k) o.F(i, j, k) = temp1[k];
        }
    });
}

// erranalysis (solution.f90:77-130)
void erranalysis(Ora& o) {
    double t1 = 0.0, t2 = 0.0;
    for (int i = 2; i <= o.Nx - 1; ++i)
        for (int j = 2; j <= o.Ny - 1; ++j) {
            size_t id = o.IX(i, j);
            double du = o.u[id] - o.u0[id], dv = o.v[id] - o.v0[id];
            t1 = t1 + du * du + dv * dv;
            t2 = t2 + o.u[id] * o.u[id] + o.v[id] * o.v[id];
        }
    t1 = std::sqrt(t1);
    t2 = std::sqrt(t2);
    o.err = t1 / (t2 + 1e-30);
}

// delta kernel, smooth=1 branch (boundary_condition.f90:1580-1600)
double phi(double disr) {
    if (std::fabs(disr) <= 0.5)
        return 0.375 + 0.03125 * PAI - 0.25 * disr * disr;
    if (std::fabs(disr) <= 1.5 && std::fabs(disr) >= 0.5)
        return 0.25 + 0.125 * (1.0 - disr) * std::sqrt(-2.0 + 8.0 * disr - 4.0 * disr * disr) -
               0.125 * std::asin(std::sqrt(2.0) * (disr - 1.0));
    if (std::fabs(disr) <= 2.5 && std::fabs(disr) >= 1.5)
        return 1.0625 - 0.015625 * PAI - 0.75 * disr + 0.125 * disr * disr +
               0.0625 * (disr - 2.0) * std::sqrt(-14.0 + 16.0 * disr - 4.0 * disr * disr) +
               0.0625 * std::asin(std::sqrt(2.0) * (disr - 2.0));
    return 0.0;
}

// LU with partial pivoting and solve, the algorithm class of cusolverDnDgetrf /
// Dgetrs called at boundary_condition.f90:1632-1638 (A is n x n row-major).
bool lu_solve(std::vector<double>& A, int n, std::vector<double>& b1, std::vector<double>& b2) {
    std::vector<int> piv(n);
    for (int k = 0; k < n; ++k) {
        int p = k;
        double mx = std::fabs(A[(size_t)k * n + k]);
        for (int i = k + 1; i < n; ++i) {
            double a = std::fabs(A[(size_t)i * n + k]);
            if (a > mx) { mx = a; p = i; }
        }
        piv[k] = p;
        if (A[(size_t)p * n + k] == 0.0) return false;
        if (p != k)
            for (int j = 0; j < n; ++j) std::swap(A[(size_t)k * n + j], A[(size_t)p * n + j]);
        double pk = A[(size_t)k * n + k];
        for (int i = k + 1; i < n; ++i) A[(size_t)i * n + k] = A[(size_t)i * n + k] / pk;
        for (int i = k + 1; i < n; ++i) {
            double lik = A[(size_t)i * n + k];
            if (lik == 0.0) continue;
            double* ri = &A[(size_t)i * n];
            const double* rk = &A[(size_t)k * n];
            for (int j = k + 1; j < n; ++j) ri[j] = ri[j] - lik * rk[j];
        }
    }
    for (std::vector<double>* b : {&b1, &b2}) {
        std::vector<double>& x = *b;
        for (int k = 0; k < n; ++k)
            if (piv[k] != k) std::swap(x[k], x[piv[k]]);
        for (int i = 0; i < n; ++i) {
            double sum = x[i];
            for (int j = 0; j < i; ++j) sum = sum - A[(size_t)i * n + j] * x[j];
            x[i] = sum;
        }
        for (int i = n - 1; i >= 0; --i) {
            double sum = x[i];
            for (int j = i + 1; j < n; ++j) sum = sum - A[(size_t)i * n + j] * x[j];
            x[i] = sum / A[(size_t)i * n + i];
        }
    }
    return true;
}

// immersed_boundary_Wu (boundary_condition.f90:1512-1736), smooth=1, with the
// dense delta matrices evaluated sparsely: entries outside a segment's box are
// exact zeros of the dense loop, and every sum keeps the dense ascending order.
int immersed_boundary_wu(Ora& o) {
    const int nseg = o.nseg, nb = (int)o.ap_i.size();
    if (nseg == 0) return 0;
    std::vector<double> ub(nseg), vb(nseg);
    for (int w = 0; w < o.W; ++w) {
        int ss = o.sstart[w], ps = o.pstart[w];
        double sn = std::sin(o.angle[w]), cs = std::cos(o.angle[w]);
        for (int i = ss; i < ss + o.pts[w] - 1; ++i) {
            int p = ps + (i - ss);
            double xs = o.xb0[p + 1] + o.xb0[p], ys = o.yb0[p + 1] + o.yb0[p];
            ub[i] = o.UU * (-(o.omega[w] * sn * 0.5 * xs) + o.omega[w] * cs * 0.5 * ys + o.sau[w]) +
                    o.extra_v[w];
            vb[i] = o.UU * (-(o.omega[w] * cs * 0.5 * xs) - o.omega[w] * sn * 0.5 * ys + o.sbv[w]);
        }
    }
    // sparse xx1 rows (per segment, ascending band index) and columns
    // (per band node, ascending segment index)
    std::vector<std::vector<std::pair<int, double>>> rows(nseg), cols(nb);
    for (int k = 0; k < nseg; ++k) {
        double x2 = o.xb2[k], y2 = o.yb2[k];
        int ic = (int)((x2 - o.ox) / o.scale + 1.0), jc = (int)((y2 - o.oy) / o.scale + 1.0);
        for (int i = std::max(1, ic - 4); i <= std::min(o.Nx, ic + 4); ++i) {
            double x0 = o.ox + o.scale * (double)(i - 1);
            double dxr = std::fabs((x0 - x2) / o.scale);
            if (dxr > 2.5) continue;
            double k1 = phi(dxr);
            for (int j = std::max(1, jc - 4); j <= std::min(o.Ny, jc + 4); ++j) {
                double y0 = o.oy + o.scale * (double)(j - 1);
                double dyr = std::fabs((y0 - y2) / o.scale);
                if (dyr > 2.5) continue;
                int b = o.bandidx[o.IX(i, j)];
                if (b < 0) return -2;  // box node outside the band: impossible by construction
                double k2 = phi(dyr);
                rows[k].push_back({b, k1 * k2});
            }
        }
        std::sort(rows[k].begin(), rows[k].end());
        for (auto& pr : rows[k]) cols[pr.first].push_back({k, pr.second});
    }
    std::vector<double> ustar(nb), vstar(nb);
    for (int b = 0; b < nb; ++b) {
        size_t id = o.IX(o.ap_i[b], o.ap_j[b]);
        ustar[b] = o.u[id];
        vstar[b] = o.v[id];
    }
    // A = xx1 * xx2, ascending band index (cublasDgemm, :1619)
    std::vector<double> A((size_t)nseg * nseg, 0.0);
    for (int b = 0; b < nb; ++b)
        for (auto& pk : cols[b])
            for (auto& pl : cols[b])
                A[(size_t)pk.first * nseg + pl.first] =
                    A[(size_t)pk.first * nseg + pl.first] + pk.second * (pl.second * o.arc[pl.first]);
    std::vector<double> c1(nseg), c2(nseg);
    for (int k = 0; k < nseg; ++k) {
        double bu = 0.0, bv = 0.0;
        for (auto& pr : rows[k]) {
            bu = bu + pr.second * ustar[pr.first];
            bv = bv + pr.second * vstar[pr.first];
        }
        c1[k] = ub[k] - bu;
        c2[k] = vb[k] - bv;
    }
    std::vector<double> r1 = c1, r2 = c2;
    if (!lu_solve(A, nseg, c1, c2)) return -3;
    std::vector<double> glx(nb), gly(nb);
    for (int b = 0; b < nb; ++b) {
        double sx = 0.0, sy = 0.0;
        for (auto& pk : cols[b]) {
            double x2v = pk.second * o.arc[pk.first];
            sx = sx + x2v * c1[pk.first];
            sy = sy + x2v * c2[pk.first];
        }
        glx[b] = sx;
        gly[b] = sy;
    }
    // no-slip residual diagnostic |X du - r| / |r|
    double rn = 0.0, en = 0.0;
    for (int k = 0; k < nseg; ++k) {
        double ax = 0.0, ay = 0.0;
        for (auto& pr : rows[k]) { ax += pr.second * glx[pr.first]; ay += pr.second * gly[pr.first]; }
        en += (ax - r1[k]) * (ax - r1[k]) + (ay - r2[k]) * (ay - r2[k]);
        rn += r1[k] * r1[k] + r2[k] * r2[k];
    }
    o.ibm_resid = std::sqrt(en) / (std::sqrt(rn) + 1e-300);
    for (int b = 0; b < nb; ++b) {
        size_t id = o.IX(o.ap_i[b], o.ap_j[b]);
        o.u[id] = ustar[b] + glx[b];
        o.v[id] = vstar[b] + gly[b];
        o.gfx[id] = 2.0 * o.rho[id] * glx[b];
        o.gfy[id] = 2.0 * o.rho[id] * gly[b];
    }
    // per-wing force and moment on the host (:1661-1675)
    std::fill(o.wing_force.begin(), o.wing_force.end(), 0.0);
    std::fill(o.wing_moment.begin(), o.wing_moment.end(), 0.0);
    for (int b = 0; b < nb; ++b) {
        int w = o.ap_w[b];
        size_t id = o.IX(o.ap_i[b], o.ap_j[b]);
        double t1 = 2.0 * o.rho[id] * glx[b];
        double t2 = 2.0 * o.rho[id] * gly[b];
        o.wing_force[w * 2 + 0] = o.wing_force[w * 2 + 0] - t1;
        o.wing_force[w * 2 + 1] = o.wing_force[w * 2 + 1] - t2;
        double x0 = (o.ox + o.scale * (double)(o.ap_i[b] - 1) -
                     (o.c.xc + o.c.wing_x_origin + (double)w * o.c.wing_x_spacing + o.sa[w])) /
                        o.scale -
                    o.extra_pos[w];
        double y0 = (o.oy + o.scale * (double)(o.ap_j[b] - 1) - (o.c.yc + o.c.wing_y_origin + o.sb[w])) /
                    o.scale;
        o.wing_moment[w] = o.wing_moment[w] - x0 * t2 + y0 * t1;
    }
    return 0;
}

// boundary_condition1, live part (boundary_condition.f90:288-858)
void outer_bc(Ora& o) {
    const int Nx = o.Nx, Ny = o.Ny;
    const double cs = (double)std::sqrt(3.0f) / 3.0;  // sqrt of a REAL(4) literal (:303)
    auto edge_f = [&](int ie, int je, int in, int jn) {
        // f(edge) = M^-1 [ m_eq(edge) + (1-s)(M f0(nbr) - m_eq(nbr)) ], m_eq with j^2/rho
        double temp[10], temp1[10], temp2[10], temp3[10];
        double rh = o.rho[o.IX(ie, je)];
        double jx = rh * o.u[o.IX(ie, je)];
        double jy = rh * o.v[o.IX(ie, je)];
        temp1[1] = rh;
        temp1[2] = -2.0 * rh + 3.0 * (jx * jx + jy * jy) / rh;
        temp1[3] = rh - 3.0 * (jx * jx + jy * jy) / rh;
        temp1[4] = jx; temp1[5] = -jx; temp1[6] = jy; temp1[7] = -jy;
        temp1[8] = (jx * jx - jy * jy) / rh;
        temp1[9] = (jx * jy) / rh;
        rh = o.rho[o.IX(in, jn)];
        jx = rh * o.u[o.IX(in, jn)];
        jy = rh * o.v[o.IX(in, jn)];
        temp2[1] = rh;
        temp2[2] = -2.0 * rh + 3.0 * (jx * jx + jy * jy) / rh;
        temp2[3] = rh - 3.0 * (jx * jx + jy * jy) / rh;
        temp2[4] = jx; temp2[5] = -jx; temp2[6] = jy; temp2[7] = -jy;
        temp2[8] = (jx * jx - jy * jy) / rh;
        temp2[9] = (jx * jy) / rh;
        for (int k = 1; k <= 9; ++k) temp[k] = o.F0(in, jn, k);
        matmulvoc(temp3, o.matm, temp);
        for (int k = 1; k <= 9; ++k) temp3[k] = temp1[k] + (1.0 - o.s[k]) * (temp3[k] - temp2[k]);
        matmulvoc(temp, o.minv, temp3);
        for (int k = 1; k <= 9; ++k) o.F(ie, je, k) = temp[k];
    };
    std::vector<double> trho(Ny + 1), tu(Ny + 1), tv(Ny + 1);
    // left (:408-481)
    for (int j = 1; j <= Ny; ++j) {
        trho[j] = o.rho[o.IX(1, j)]; tu[j] = o.u[o.IX(1, j)]; tv[j] = o.v[o.IX(1, j)];
    }
    for (int j = 2; j <= Ny - 1; ++j) {
        double rhox = (-3.0 * trho[j] + 4.0 * o.rho[o.IX(2, j)] - o.rho[o.IX(3, j)]) * 0.5;
        double ux = (-3.0 * tu[j] + 4.0 * o.u[o.IX(2, j)] - o.u[o.IX(3, j)]) * 0.5;
        double vx = (-3.0 * tv[j] + 4.0 * o.v[o.IX(2, j)] - o.v[o.IX(3, j)]) * 0.5;
        double lx1 = (tu[j] - cs) * (cs * cs * rhox - cs * trho[j] * ux);
        double lx2 = (tu[j] < 0.0) ? tu[j] * vx : 0.0;
        double lx3 = 0.0;
        size_t id = o.IX(1, j);
        o.rho[id] = o.rho[id] - (lx1 + lx3) * 1.5;
        o.u[id] = o.u[id] + (lx1 - lx3) / (2.0 * cs * o.rho[id]);
        o.v[id] = o.v[id] - lx2;
    }
    for (int j = 2; j <= Ny - 1; ++j) edge_f(1, j, 2, j);
    // right (:489-565)
    for (int j = 1; j <= Ny; ++j) {
        trho[j] = o.rho[o.IX(Nx, j)]; tu[j] = o.u[o.IX(Nx, j)]; tv[j] = o.v[o.IX(Nx, j)];
    }
    for (int j = 2; j <= Ny - 1; ++j) {
        double rhox = (3.0 * trho[j] - 4.0 * o.rho[o.IX(Nx - 1, j)] + o.rho[o.IX(Nx - 2, j)]) * 0.5;
        double ux = (3.0 * tu[j] - 4.0 * o.u[o.IX(Nx - 1, j)] + o.u[o.IX(Nx - 2, j)]) * 0.5;
        double vx = (3.0 * tv[j] - 4.0 * o.v[o.IX(Nx - 1, j)] + o.v[o.IX(Nx - 2, j)]) * 0.5;
        double lx1 = 0.0;
        double lx2 = (tu[j] >= 0.0) ? tu[j] * vx : 0.0;
        double lx3 = (tu[j] + cs) * (cs * cs * rhox + cs * trho[j] * ux);
        size_t id = o.IX(Nx, j);
        o.rho[id] = o.rho[id] - (lx1 + lx3) * 1.5;
        o.u[id] = o.u[id] + (lx1 - lx3) / (2.0 * cs * o.rho[id]);
        o.v[id] = o.v[id] - lx2;
    }
    for (int j = 2; j <= Ny - 1; ++j) edge_f(Nx, j, Nx - 1, j);
    // top (:655-708): rho from the row below, zero velocity
    for (int i = 1; i <= Nx; ++i) {
        size_t id = o.IX(i, Ny);
        o.rho[id] = o.rho[o.IX(i, Ny - 1)];
        o.u[id] = 0.0;
        o.v[id] = 0.0;
        edge_f(i, Ny, i, Ny - 1);
    }
    // bottom (:782-835)
    for (int i = 1; i <= Nx; ++i) {
        size_t id = o.IX(i, 1);
        o.rho[id] = o.rho[o.IX(i, 2)];
        o.u[id] = 0.0;
        o.v[id] = 0.0;
        edge_f(i, 1, i, 2);
    }
}

// evolution (solution.f90:272-422)
int evolution(Ora& o, int64_t cycle, double* force_row) {
    o.time = (double)(cycle - 1) * (o.scale * o.UU);
    if (o.time >= 0.0) {
        if (mode(o) != 0) return -1;
        move_boundary(o);
    }
    streaming(o);
    physical_variables(o);
    int rc = immersed_boundary_wu(o);
    if (rc != 0) return rc;
    colission(o);
    const int W = o.W;
    for (int w = 0; w < W; ++w) {
        o.wing_force[w * 2 + 0] = 2.0 * o.wing_force[w * 2 + 0] / (o.UU * o.UU * (1.0 / o.scale));
        o.wing_force[w * 2 + 1] = 2.0 * o.wing_force[w * 2 + 1] / (o.UU * o.UU * (1.0 / o.scale));
        o.wing_moment[w] =
            -(2.0 * o.wing_moment[w] / (o.UU * o.UU * (1.0 / (o.scale * o.scale))));
    }
    double fx = 0.0, fy = 0.0, mt = 0.0;
    for (int w = 0; w < W; ++w) { fx = fx + o.wing_force[w * 2]; fy = fy + o.wing_force[w * 2 + 1]; }
    for (int w = 0; w < W; ++w) mt = mt + o.wing_moment[w];
    std::vector<double> row(4 + 12 * W, 0.0);
    row[0] = o.time;
    int col = 1;
    for (int w = 0; w < W; ++w) {
        row[col] = o.wing_force[w * 2]; row[col + 1] = o.wing_force[w * 2 + 1];
        row[col + 2] = o.wing_moment[w];
        col += 3;
    }
    row[col] = fx; row[col + 1] = fy; row[col + 2] = mt;
    col += 3;
    for (int w = 0; w < W; ++w) {
        row[col] = o.c.wing_x_origin + (double)w * o.c.wing_x_spacing + o.sa[w] +
                   o.extra_s[w] / (1.0 / o.scale);
        row[col + 1] = o.sau[w];
        row[col + 2] = o.saac[w];
        row[col + 3] = o.c.wing_y_origin + o.sb[w];
        row[col + 4] = o.sbv[w];
        row[col + 5] = o.sbac[w];
        row[col + 6] = o.angle[w];
        row[col + 7] = o.omega[w];
        row[col + 8] = o.omgac[w];
        col += 9;
    }
    o.row_len = col;
    for (int c = 0; c < col; ++c) o.sum_row[c] = o.sum_row[c] + row[c];
    o.sample_count += 1;
    if (force_row) std::memcpy(force_row, row.data(), sizeof(double) * col);
    outer_bc(o);
    return 0;
}

// move_mesh single-rank path (move_mesh.f90:29-58 for dr=+1, :185-214 for dr=-1)
void move_mesh(Ora& o, int dr) {
    const int Nx = o.Nx, Ny = o.Ny;
    int klo = (dr == 1) ? 1 : 2, khi = (dr == 1) ? Nx - 1 : Nx, src = (dr == 1) ? 1 : -1;
    for (int j = 1; j <= Ny; ++j)
        for (int k = klo; k <= khi; ++k) {
            for (int q = 1; q <= 9; ++q) o.F0(k, j, q) = o.F(k + src, j, q);
            o.u0[o.IX(k, j)] = o.u[o.IX(k + src, j)];
            o.v0[o.IX(k, j)] = o.v[o.IX(k + src, j)];
            o.pre[o.IX(k, j)] = o.rho[o.IX(k + src, j)];
        }
    for (int j = 1; j <= Ny; ++j)
        for (int k = klo; k <= khi; ++k) {
            for (int q = 1; q <= 9; ++q) o.F(k, j, q) = o.F0(k, j, q);
            o.u[o.IX(k, j)] = o.u0[o.IX(k, j)];
            o.v[o.IX(k, j)] = o.v0[o.IX(k, j)];
            o.rho[o.IX(k, j)] = o.pre[o.IX(k, j)];
        }
}

}  // namespace

extern "C" {

void* ora_create(const OraConfig* cfg, const double* markers_xy, const int32_t* points_per_wing,
                 int32_t nthreads) {
    if (!cfg || cfg->nx < 5 || cfg->ny < 5 || cfg->wing_count < 0) return nullptr;
    Ora* o = new Ora();
    o->c = *cfg;
    o->nthreads = nthreads > 0 ? nthreads : 1;
    o->Nx = cfg->nx; o->Ny = cfg->ny; o->N = o->Nx * o->Ny;
    o->scale = cfg->scale; o->UU = cfg->uu; o->ox = cfg->ox; o->oy = cfg->oy;
    // ini_mesh.f90:30-31, 59-67
    o->niu = o->UU * (1.0 / o->scale) / cfg->re;
    o->tau = 3.0 * o->niu + 0.5;
    for (int k = 1; k <= 9; ++k) o->s[k] = cfg->s[k - 1];
    if (o->s[8] <= 0.0) o->s[8] = 1.0 / o->tau;
    if (o->s[9] <= 0.0) o->s[9] = 1.0 / o->tau;
    d2q9model(*o);
    set_matm(*o);
    const size_t N = (size_t)o->N;
    o->f.assign(9 * N, 0.0); o->f0.assign(9 * N, 0.0);
    o->rho.assign(N, 1.0); o->u.assign(N, o->UU); o->v.assign(N, 0.0);
    o->u0.assign(N, o->UU); o->v0.assign(N, 0.0); o->pre.assign(N, 1.0 / 3.0);
    o->gfx.assign(N, 0.0); o->gfy.assign(N, 0.0);
    o->body.assign(N, 0); o->bandidx.assign(N, -1);
    // init (solution.f90:44-61): f = f0 = feq(rho0=1, u=UU, v=0) everywhere
    for (int j = 1; j <= o->Ny; ++j)
        for (int i = 1; i <= o->Nx; ++i)
            for (int k = 1; k <= 9; ++k) {
                double fe = d2q9feq(*o, 1.0, o->UU, 0.0, k);
                o->F(i, j, k) = fe;
                o->F0(i, j, k) = fe;
            }
    const int W = cfg->wing_count;
    o->W = W;
    o->ncol = 1 + 9 * W;
    o->pts.resize(W); o->pstart.resize(W); o->sstart.resize(W);
    int np = 0, ns = 0;
    for (int w = 0; w < W; ++w) {
        if (points_per_wing[w] < 2) { delete o; return nullptr; }
        o->pts[w] = points_per_wing[w];
        o->pstart[w] = np; o->sstart[w] = ns;
        np += points_per_wing[w]; ns += points_per_wing[w] - 1;
    }
    o->npts = np; o->nseg = ns;
    o->xb0.resize(np); o->yb0.resize(np); o->xb1.assign(np, 0); o->yb1.assign(np, 0);
    o->xb2.assign(ns, 0); o->yb2.assign(ns, 0); o->arc.assign(ns, 0); o->seg_wing.resize(ns);
    // read_boundary (airfoil.f90:214-241)
    for (int p = 0; p < np; ++p) {
        o->xb0[p] = markers_xy[2 * p] + (cfg->xc - 0.0);
        o->yb0[p] = markers_xy[2 * p + 1] + (cfg->yc - 0.0);
    }
    for (int w = 0; w < W; ++w)
        for (int i0 = 0; i0 < o->pts[w] - 1; ++i0) {
            int p = o->pstart[w] + i0;
            double ddx = markers_xy[2 * (p + 1)] - markers_xy[2 * p];
            double ddy = markers_xy[2 * (p + 1) + 1] - markers_xy[2 * p + 1];
            o->arc[o->sstart[w] + i0] = std::sqrt(ddx * ddx + ddy * ddy) / o->scale;
            o->seg_wing[o->sstart[w] + i0] = w;
        }
    auto z = [W](std::vector<double>& v) { v.assign(W, 0.0); };
    z(o->angle); z(o->omega); z(o->omgac); z(o->sa); z(o->sau); z(o->saac); z(o->sb);
    z(o->sbv); z(o->sbac); z(o->rel_v); z(o->rel_s); z(o->rel_pos); z(o->extra_v);
    z(o->extra_s); z(o->extra_pos); z(o->wing_moment);
    o->wing_force.assign(2 * W, 0.0);
    o->sum_row.assign(4 + 12 * W, 0.0);
    o->stream_start.assign(o->ncol, 0.0);
    o->stream_target.assign(o->ncol, 0.0);
    return o;
}

void ora_destroy(void* h) { delete static_cast<Ora*>(h); }

// load_motion_table + build_motion_step_table (mode.f90:104-178, 388-412)
int ora_set_motion_table(void* h, const double* rows, int64_t nrows, int32_t ncols) {
    Ora& o = *static_cast<Ora*>(h);
    if (ncols != o.ncol || nrows < 1) return -1;
    o.table.assign(rows, rows + (size_t)nrows * ncols);
    o.table_rows = nrows;
    for (int64_t i = 1; i < nrows; ++i)
        if (o.table[(size_t)i * ncols] < o.table[(size_t)(i - 1) * ncols]) return -2;
    o.motion_end_time = o.table[(size_t)(nrows - 1) * ncols];
    o.motion_index = 1;
    double dt = o.scale * o.UU;
    o.motion_dt = dt;
    o.step_rows = (int64_t)((o.motion_end_time + 1.0e-12) / dt) + 1;
    o.step_table.assign((size_t)o.step_rows * ncols, 0.0);
    std::vector<double> row(ncols);
    for (int64_t i = 1; i <= o.step_rows; ++i) {
        double t = (double)(i - 1) * dt;
        lookup_motion_row(o, t, row.data());
        std::memcpy(&o.step_table[(size_t)(i - 1) * ncols], row.data(), sizeof(double) * ncols);
    }
    return 0;
}

int ora_set_stream_rows(void* h, const double* start_row, const double* target_row) {
    Ora& o = *static_cast<Ora*>(h);
    o.stream_start.assign(start_row, start_row + o.ncol);
    o.stream_target.assign(target_row, target_row + o.ncol);
    o.stream_ready = true;
    return 0;
}

int ora_step(void* h, int64_t n, double* force_row) {
    Ora& o = *static_cast<Ora*>(h);
    if (n >= 2) erranalysis(o);
    int rc = evolution(o, n, force_row);
    if (rc != 0) return rc;
    // lattice shift when the first wing has drifted one column (main.f90:393-411)
    if (o.W > 0 && o.rel_pos[0] >= 1.0) {
        move_mesh(o, 1);
        o.rel_pos[0] -= 1.0;
        update_body_extra(o);
        o.movenum += 1;
    } else if (o.W > 0 && o.rel_pos[0] <= -1.0) {
        move_mesh(o, -1);
        o.rel_pos[0] += 1.0;
        update_body_extra(o);
        o.movenum -= 1;
    }
    return 0;
}

double ora_err(void* h) {
    Ora& o = *static_cast<Ora*>(h);
    erranalysis(o);
    return o.err;
}

double ora_tau(void* h) { return static_cast<Ora*>(h)->tau; }

int ora_get_field(void* h, int32_t which, double* out) {
    Ora& o = *static_cast<Ora*>(h);
    const size_t N = (size_t)o.N;
    const std::vector<double>* src = nullptr;
    switch (which) {
        case 0: src = &o.rho; break;
        case 1: src = &o.u; break;
        case 2: src = &o.v; break;
        case 3: src = &o.pre; break;
        case 4: src = &o.u0; break;
        case 5: src = &o.v0; break;
        case 6: src = &o.gfx; break;
        case 7: src = &o.gfy; break;
        default: break;
    }
    if (src) { std::memcpy(out, src->data(), N * sizeof(double)); return 0; }
    if (which >= 100 && which < 109) {
        std::memcpy(out, &o.f[(size_t)(which - 100) * N], N * sizeof(double));
        return 0;
    }
    if (which >= 200 && which < 209) {
        std::memcpy(out, &o.f0[(size_t)(which - 200) * N], N * sizeof(double));
        return 0;
    }
    return -1;
}

int ora_set_f(void* h, const double* f) {
    Ora& o = *static_cast<Ora*>(h);
    std::memcpy(o.f.data(), f, o.f.size() * sizeof(double));
    return 0;
}

int ora_get_band(void* h, int32_t* n, int32_t* ij_wing, int32_t cap) {
    Ora& o = *static_cast<Ora*>(h);
    int nb = (int)o.ap_i.size();
    *n = nb;
    if (!ij_wing) return 0;
    for (int b = 0; b < nb && b < cap; ++b) {
        ij_wing[3 * b] = o.ap_i[b]; ij_wing[3 * b + 1] = o.ap_j[b]; ij_wing[3 * b + 2] = o.ap_w[b] + 1;
    }
    return nb <= cap ? 0 : -1;
}

int ora_get_markers(void* h, double* xb1, double* yb1, double* xb2, double* yb2) {
    Ora& o = *static_cast<Ora*>(h);
    if (xb1) std::memcpy(xb1, o.xb1.data(), o.npts * sizeof(double));
    if (yb1) std::memcpy(yb1, o.yb1.data(), o.npts * sizeof(double));
    if (xb2) std::memcpy(xb2, o.xb2.data(), o.nseg * sizeof(double));
    if (yb2) std::memcpy(yb2, o.yb2.data(), o.nseg * sizeof(double));
    return 0;
}

int ora_get_sums(void* h, double* sum_row, int32_t* sample_count, int32_t* row_len) {
    Ora& o = *static_cast<Ora*>(h);
    if (sum_row) std::memcpy(sum_row, o.sum_row.data(), o.sum_row.size() * sizeof(double));
    if (sample_count) *sample_count = o.sample_count;
    if (row_len) *row_len = o.row_len;
    return 0;
}

void ora_reset_sums(void* h) {
    Ora& o = *static_cast<Ora*>(h);
    std::fill(o.sum_row.begin(), o.sum_row.end(), 0.0);
    o.sample_count = 0;
    o.row_len = 0;
}

int ora_stream_row(void* h, double t, double* row) {
    Ora& o = *static_cast<Ora*>(h);
    if (!o.stream_ready) return -1;
    lookup_stream_row(o, t, row);
    return 0;
}

// build_stream_target_row (mode.f90:287-325); delta_row holds t then 3 values per wing.
int ora_build_stream_target_row(void* h, const double* start_row, double target_time,
                                const double* delta_row, double* target_row) {
    Ora& o = *static_cast<Ora*>(h);
    double dt = target_time - start_row[0];
    if (dt < -1.0e-12) return -1;
    for (int c = 0; c < o.ncol; ++c) target_row[c] = start_row[c];
    target_row[0] = target_time;
    for (int w = 0; w < o.W; ++w) {
        int col = 1 + w * 9, dcol = 1 + w * 3;
        for (int t = 0; t < 3; ++t) {
            int cc = col + 3 * t;
            triplet(start_row[cc], start_row[cc + 1], start_row[cc + 1] + delta_row[dcol + t], dt,
                    std::max(dt, 0.0), &target_row[cc], &target_row[cc + 1], &target_row[cc + 2]);
        }
    }
    return 0;
}

void ora_interpolate_triplet(double s0, double v0, double v1, double dt, double local_t, double* s,
                             double* v, double* a) {
    triplet(s0, v0, v1, dt, local_t, s, v, a);
}

double ora_delta_phi(double r) { return phi(std::fabs(r)); }

void ora_inverse_m(double* minv81) {
    Ora o;
    set_matm(o);
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) minv81[i * 9 + j] = o.minv[i + 1][j + 1];
}

int ora_move_mesh(void* h, int32_t dr) {
    Ora& o = *static_cast<Ora*>(h);
    if (dr != 1 && dr != -1) return -1;
    move_mesh(o, dr);
    o.movenum += dr;
    return 0;
}

double ora_ibm_residual(void* h) { return static_cast<Ora*>(h)->ibm_resid; }

}  // extern "C"
