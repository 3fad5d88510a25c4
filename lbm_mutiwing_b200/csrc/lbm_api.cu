// C ABI and host-side orchestration: set-up (ini_mesh, init, read_boundary),
// motion tables (mode.f90), the step sequence of evolution and its
// force-row bookkeeping, field export and the lattice shift.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <queue>
#include <string>
#include <vector>

#include <cuda.h>

#include "../../include/lbm_mutiwing.h"
#include "lbm_kernels.h"

namespace lbm {

// nizhen (solution.f90:1474-1529): Gauss-Jordan inverse of M as the reference
// computes it, so the plain path multiplies by the same M^-1 entries.
static void gauss_jordan_inverse(double out[81]) {
    double a[10][10], b1[10][10];
    for (int i = 1; i <= 9; ++i)
        for (int j = 1; j <= 9; ++j) { a[i][j] = mrt_m(i - 1, j - 1); b1[i][j] = (i == j) ? 1.0 : 0.0; }
    const int Nm = 9;
    double temp, mik;
    for (int k = 1; k <= Nm - 1; ++k) {
        int ik = k;
        temp = std::fabs(a[ik][k]);
        for (int i = k; i <= Nm; ++i)
            if (std::fabs(a[i][k]) > std::fabs(temp)) { temp = std::fabs(a[i][k]); ik = i; }
        for (int j = 1; j <= Nm; ++j) {
            std::swap(a[ik][j], a[k][j]);
            std::swap(b1[ik][j], b1[k][j]);
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
    for (int j = 1; j <= Nm; ++j) b1[Nm][j] = b1[Nm][j] / temp;
    for (int i = 0; i < 9; ++i)
        for (int j = 0; j < 9; ++j) out[i * 9 + j] = b1[i + 1][j + 1];
}

// Reverse Cuthill-McKee order of one wing's segments on the graph "midpoints
// within 7.1 lattice spacings" -- a superset of the pairs whose 6 x 6 support
// boxes can overlap (|dx|, |dy| <= 5 spacings), invariant under the wing's
// rigid motion.  Returns the order and the half bandwidth.
static int rcm_order(const std::vector<double>& mx, const std::vector<double>& my, double spacing,
                     std::vector<int>& order) {
    const int n = (int)mx.size();
    const double r2 = (7.1 * spacing) * (7.1 * spacing);
    std::vector<std::vector<int>> adj(n);
    for (int a = 0; a < n; ++a)
        for (int b = a + 1; b < n; ++b) {
            double dx = mx[a] - mx[b], dy = my[a] - my[b];
            if (dx * dx + dy * dy <= r2) { adj[a].push_back(b); adj[b].push_back(a); }
        }
    std::vector<int> deg(n);
    for (int a = 0; a < n; ++a) deg[a] = (int)adj[a].size();
    std::vector<char> seen(n, 0);
    std::vector<int> cm;
    cm.reserve(n);
    while ((int)cm.size() < n) {
        int start = -1;
        for (int a = 0; a < n; ++a)
            if (!seen[a] && (start < 0 || deg[a] < deg[start])) start = a;
        std::queue<int> q;
        q.push(start);
        seen[start] = 1;
        while (!q.empty()) {
            int a = q.front();
            q.pop();
            cm.push_back(a);
            std::vector<int> nb;
            for (int b : adj[a])
                if (!seen[b]) { seen[b] = 1; nb.push_back(b); }
            std::sort(nb.begin(), nb.end(), [&](int x, int y) { return deg[x] != deg[y] ? deg[x] < deg[y] : x < y; });
            for (int b : nb) q.push(b);
        }
    }
    order.assign(cm.rbegin(), cm.rend());
    std::vector<int> pos(n);
    for (int p = 0; p < n; ++p) pos[order[p]] = p;
    int bw = 0;
    for (int a = 0; a < n; ++a)
        for (int b : adj[a]) bw = std::max(bw, std::abs(pos[a] - pos[b]));
    return bw;
}

}  // namespace lbm

using namespace lbm;

// phase timers: move_boundary, collide-stream, band re-collision, far field,
// immersed-boundary solve, factorisation, far tiles of passes
constexpr int NPHASE = 7;

// Immersed-boundary geometry of one step: motion, markers, support boxes,
// kernel values, band list and map, and the factorised G.  It depends only
// on the motion, so the fused path builds it GEO_AHEAD steps in advance, on
// side streams, into one of GEO_SETS sets while earlier steps read theirs:
// a two-step pass reads the sets of its two steps and builds the next two.
#ifndef LBM_GEO_AHEAD
#define LBM_GEO_AHEAD 2
#endif
constexpr int GEO_AHEAD = LBM_GEO_AHEAD, GEO_SETS = 2 * GEO_AHEAD;
// steps per CUDA graph of single steps: a multiple of 2 (the two plane
// copies alternate) and of GEO_SETS, so a graph ends in the state it started
// from (graphs of passes hold one pass)
#ifndef LBM_GRAPH_STEPS
#define LBM_GRAPH_STEPS (GEO_SETS % 2 ? 2 * GEO_SETS : GEO_SETS)
#endif
constexpr int GRAPH_STEPS = LBM_GRAPH_STEPS;
static_assert(GRAPH_STEPS % 2 == 0 && GRAPH_STEPS % GEO_SETS == 0, "a graph returns to its planes and set");
struct GeoSet {
    WingMotion* wm = nullptr;
    double *xb1 = nullptr, *yb1 = nullptr, *xb2 = nullptr, *yb2 = nullptr, *kx = nullptr, *ky = nullptr;
    int *box = nullptr, *claim_cnt = nullptr, *pb = nullptr, *band_claimer = nullptr, *band_n = nullptr;
    int *band_ij = nullptr, *band_wing = nullptr, *band_map = nullptr, *ibm_flags = nullptr;
    unsigned* band_bits = nullptr;
    double *lband = nullptr, *linv = nullptr, *lq = nullptr;
    unsigned char* tile_flags = nullptr;
    int *tile_list = nullptr, *tile_n = nullptr;
};

static GeoSet geo_of(const DevState& d) {
    GeoSet g;
    g.wm = d.wm; g.xb1 = d.xb1; g.yb1 = d.yb1; g.xb2 = d.xb2; g.yb2 = d.yb2; g.kx = d.kx; g.ky = d.ky;
    g.box = d.box; g.claim_cnt = d.claim_cnt; g.pb = d.pb; g.band_claimer = d.band_claimer;
    g.band_n = d.band_n; g.band_ij = d.band_ij; g.band_wing = d.band_wing; g.band_map = d.band_map;
    g.band_bits = d.band_bits;
    g.ibm_flags = d.ibm_flags; g.lband = d.lband; g.linv = d.linv; g.lq = d.lq;
    g.tile_flags = d.tile_flags; g.tile_list = d.tile_list; g.tile_n = d.tile_n;
    return g;
}

static void use_geo(DevState& d, const GeoSet& g) {
    d.wm = g.wm; d.xb1 = g.xb1; d.yb1 = g.yb1; d.xb2 = g.xb2; d.yb2 = g.yb2; d.kx = g.kx; d.ky = g.ky;
    d.box = g.box; d.claim_cnt = g.claim_cnt; d.pb = g.pb; d.band_claimer = g.band_claimer;
    d.band_n = g.band_n; d.band_ij = g.band_ij; d.band_wing = g.band_wing; d.band_map = g.band_map;
    d.band_bits = g.band_bits;
    d.ibm_flags = g.ibm_flags; d.lband = g.lband; d.linv = g.linv; d.lq = g.lq;
    d.tile_flags = g.tile_flags; d.tile_list = g.tile_list; d.tile_n = g.tile_n;
}

struct LbmHandle {
    LbmConfig cfg{};
    std::string err;
    DevState d{};
    FusedConsts fc{};
    // fused path: three plane copies; a step or a pass goes from planes[cur]
    // to the third copy, which becomes cur (a pass writes its first step's
    // band and border values to planes[alt], which never changes), so cur
    // alternates between two copies
    int cur = 0, alt = 1;
    float* planes[3] = {nullptr, nullptr, nullptr};
    GeoSet geo[GEO_SETS];           // geometry sets (the plain path uses set 0)
    int gset = 0;                   // fused path: set of the next step
    int prio_lo = 0, prio_hi = 0;   // stream priority range of the device
    int prio_mid = 0;               // between them: geometry built ahead, far field
    int last_gset = 0;              // set of the last completed step
    bool pending[GEO_SETS] = {};    // set built on the side streams, not yet waited for
    // streams of one fused step: main (bulk kernel, band re-collision),
    // ibm (right-hand side, solve, spread, forces), bc (far field), and two
    // pairs of geometry streams used by alternate steps, so that the
    // geometry builds of consecutive steps run side by side: aux (motion,
    // markers, band list), aux2 (assembly and factorisation of G)
    // near: the near tiles of a pass
    cudaStream_t s_main = nullptr, s_ibm = nullptr, s_bc = nullptr, s_aux[2] = {}, s_aux2[2] = {}, s_near = nullptr;
    cudaEvent_t ev_ibm = nullptr, ev_main = nullptr, ev_bc = nullptr, ev_geom[GEO_SETS] = {};
    // a pass: first step's rhs, chain and far field done, step n + 1 ring
    // values written, near tiles done
    cudaEvent_t ev_rhs1 = nullptr, ev_chain1 = nullptr, ev_bc1 = nullptr, ev_ring = nullptr, ev_near = nullptr;
    cudaEvent_t ev_list[GEO_SETS] = {}, ev_fact[GEO_SETS] = {};   // a set's band list / factor done
    std::vector<void*> allocs;
    int64_t dev_bytes = 0;
    int row_len = 4;
    size_t factor_smem = 0;         // dynamic shared memory of the factorisation kernel
    double* err_partial = nullptr;
    double* err_out = nullptr;
    bool fields_valid = false, err_valid = false;
    // host copies
    std::vector<double> xb0, yb0;
    std::vector<int> ppw;
    double* pinned = nullptr;       // small pinned staging buffer
    size_t pinned_n = 0;
    double* d_rowbuf = nullptr;     // device force rows
    int rows_cap = 0;
    // motion (mode.f90)
    std::vector<double> table;
    int64_t table_rows = 0;
    int64_t motion_index = 1;
    double* d_step_table = nullptr;
    double* d_stream = nullptr;     // start row then target row
    int32_t status_seen = 0;
    // phase timers
    bool timing = false;
    std::vector<cudaEvent_t> evpool;
    size_t evused = 0;
    std::vector<std::pair<int, std::pair<size_t, size_t>>> marks;   // phase, (start ev, stop ev)
    double phase_ms[NPHASE] = {0, 0, 0, 0, 0, 0, 0};
    long long timed_steps = 0, timed_passes = 0;
    int* d_far_tiles = nullptr;     // far tiles processed while timing
    // CUDA graphs of GRAPH_STEPS single steps, and of one pass, by starting
    // planes (cur, alt) and geometry set; any change of a pointer or value
    // baked into DevState drops them
    cudaGraphExec_t gexec[3][3][GEO_SETS] = {};
    cudaGraphExec_t pexec[3][3][GEO_SETS] = {};
    // tensor maps of the three plane copies (fused path), for the tiled bulk
    // kernel (tmap_ok false keeps the kernel with global pulls) and the
    // pass kernels (passes run when pass_ok)
    CUtensorMap tmap[3], ptmap[3];
    bool tmap_ok = false, pass_ok = false;
    int* border_tiles = nullptr;    // pass tiles whose R1 meets the border
    int nborder = 0;
    double* d_out = nullptr;        // strided output fields (SAVE)
    size_t out_cap = 0;
    // Continuation state: the cycle the device counters hold after the last
    // call (-1: unknown), and, on the fused path, the cycle whose geometry
    // the last step of that call built into set gset (-1: none, or made
    // stale by a change of motion or lattice shift).  A call that continues
    // at next_cycle with a valid geometry writes no counter and builds no
    // geometry before its first step.
    int64_t next_cycle = -1;
    int64_t geo_ready = -1;
};

// Packed stepping of many fused-path handles (lbm_batch_step): one launch per
// kernel of a step covers every episode of the batch.  The streams mirror a
// handle's: bulk (low priority), far field and the two geometry streams
// (middle), main and immersed boundary (high).
struct LbmBatch {
    int device = 0;
    std::string err;
    cudaStream_t s_main = nullptr, s_bulk = nullptr, s_ibm = nullptr, s_bc = nullptr, s_aux = nullptr,
                 s_aux2 = nullptr;
    cudaEvent_t ev_start = nullptr, ev_bulk = nullptr, ev_ibm = nullptr, ev_bc = nullptr, ev_geom = nullptr,
                ev_list = nullptr, ev_fact = nullptr;
    char* d_buf = nullptr;          // device tables: episode states, block offsets, state pointers
    size_t d_cap = 0;
    char* h_buf = nullptr;          // pinned staging of the tables
    size_t h_cap = 0;
    // autotuning of the packed bulk kernel's runs per block: batch shape
    // (sorted lattice sizes) -> fastest kind, and the events that time it
    std::map<std::vector<long long>, int> bulk_kind;
    cudaEvent_t ev_tune[4] = {};
    // CUDA graphs of two packed steps, by everything their launches bake in
    // (table addresses, block offsets, bulk variant)
    std::map<std::vector<long long>, cudaGraphExec_t> graphs;
    int prio_lo = 0, prio_mid = 0, prio_hi = 0;
};

namespace {

// Graph capture and device-wide operations of different handles must not
// interleave: an allocation, a free or a device synchronisation issued by
// one thread while another thread captures a step graph invalidates that
// capture.  Every entry point that allocates, frees, synchronises the device
// or captures holds this lock (handles are otherwise independent).
std::recursive_mutex g_device_mutex;
using DeviceLock = std::lock_guard<std::recursive_mutex>;

void drop_graphs(LbmHandle* h);

int fail(LbmHandle* h, const std::string& msg) {
    if (h) h->err = msg;
    return -1;
}

int cuda_fail(LbmHandle* h, cudaError_t e, const char* where) {
    return fail(h, std::string("CUDA error in ") + where + ": " + cudaGetErrorString(e));
}

#define CK(call)                                                   \
    do {                                                           \
        cudaError_t e_ = (call);                                   \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call);     \
    } while (0)

// words of a band bit plane (one bit per pitched node index)
size_t band_bits_words(const DevState& d) { return (size_t)((d.plane + 31) / 32); }

template <class T>
int dalloc(LbmHandle* h, T** p, size_t count) {
    DeviceLock lock(g_device_mutex);
    size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t e = cudaMalloc((void**)p, bytes);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaMalloc");
    h->allocs.push_back(*p);
    h->dev_bytes += (int64_t)bytes;
    return 0;
}

DevState current(const LbmHandle* h) {
    DevState d = h->d;
    if (d.precision != 0) {
        d.gA = h->planes[h->cur];
        d.gB = h->planes[3 - h->cur - h->alt];
        use_geo(d, h->geo[h->gset]);
    }
    return d;
}
int third_planes(const LbmHandle* h) { return 3 - h->cur - h->alt; }

// The geometry of the last completed step (band list, markers).
DevState last_geometry(const LbmHandle* h) {
    DevState d = h->d;
    use_geo(d, h->geo[d.precision != 0 ? h->last_gset : 0]);
    return d;
}

// interpolate_motion_row / lookup_motion_row (mode.f90:327-386)
void lookup_motion_row(LbmHandle* h, double target, double* row) {
    const int nc = 1 + 9 * h->cfg.wing_count;
    const double tol = 1.0e-12;
    const int64_t np = h->table_rows;
    const double* T = h->table.data();
    auto rowp = [&](int64_t i) { return T + (size_t)(i - 1) * nc; };
    if (target <= rowp(1)[0] + tol) {
        h->motion_index = 1;
        std::memcpy(row, rowp(1), sizeof(double) * nc);
        row[0] = target;
        return;
    }
    if (target >= rowp(np)[0] - tol) {
        h->motion_index = np;
        std::memcpy(row, rowp(np), sizeof(double) * nc);
        row[0] = target;
        return;
    }
    h->motion_index = std::max<int64_t>(1, std::min<int64_t>(h->motion_index, np - 1));
    while (h->motion_index > 1 && target <= rowp(h->motion_index)[0] + tol) h->motion_index -= 1;
    while (h->motion_index < np - 1 && target > rowp(h->motion_index + 1)[0] + tol) h->motion_index += 1;
    const double* r1 = rowp(h->motion_index);
    const double* r2 = rowp(h->motion_index + 1);
    double t1 = r1[0], t2 = r2[0], dt = t2 - t1;
    if (std::fabs(dt) <= 1.0e-14) {
        std::memcpy(row, r2, sizeof(double) * nc);
        row[0] = target;
        return;
    }
    double ratio = (target - t1) / dt;
    ratio = std::min(std::max(ratio, 0.0), 1.0);
    for (int c = 0; c < nc; ++c) row[c] = r1[c] + ratio * (r2[c] - r1[c]);
    row[0] = target;
}

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
void triplet(double s0, double v0, double v1, double dt, double lt, double* s, double* v, double* a) {
    double dv = v1 - v0;
    if (dt <= 1.0e-14) {
        *s = (v0 + dv) * lt + s0;
        *v = v0 + dv;
        *a = 0.0;
        return;
    }
    double x = lt / dt;
    *s = dv * dt * smooth_r(x) + v0 * lt + s0;
    *v = dv * smooth_h(x) + v0;
    *a = dv / dt * smooth_d(x);
}

int init_state(LbmHandle* h) {
    DevState d = current(h);
    const size_t N = (size_t)d.plane;
    if (d.precision == 0) {
        // f = f0 = feq(1, UU, 0); rho = 1, u = u0 = UU, v = 0, pre = 1/3 (solution.f90:44-61)
        std::vector<double> fe(9), buf(N);
        for (int k = 0; k < 9; ++k) {
            double eu = (double)ex(k) * d.uu + (double)ey(k) * 0.0;
            double utwo = d.uu * d.uu + 0.0 * 0.0;
            fe[k] = weight(k) * 1.0 * (1.0 + 3.0 * eu + 4.5 * eu * eu - 1.5 * utwo);
        }
        for (int k = 0; k < 9; ++k) {
            std::fill(buf.begin(), buf.end(), fe[k]);
            CK(cudaMemcpy(d.f + k * N, buf.data(), N * sizeof(double), cudaMemcpyHostToDevice));
            CK(cudaMemcpy(d.f0 + k * N, buf.data(), N * sizeof(double), cudaMemcpyHostToDevice));
        }
        auto fill = [&](double* p, double v) -> int {
            std::fill(buf.begin(), buf.end(), v);
            CK(cudaMemcpy(p, buf.data(), N * sizeof(double), cudaMemcpyHostToDevice));
            return 0;
        };
        if (fill(d.rho, 1.0) || fill(d.u, d.uu) || fill(d.u0, d.uu) || fill(d.v, 0.0) || fill(d.v0, 0.0) ||
            fill(d.pre, 1.0 / 3.0) || fill(d.gfx, 0.0) || fill(d.gfy, 0.0))
            return -1;
    } else {
        h->cur = 0;
        h->alt = 1;
        d = current(h);
        launch_fused_init(d, h->s_main);
        CK(cudaGetLastError());
    }
    std::vector<int> em(N, BAND_EMPTY);
    for (int s = 0; s < GEO_SETS; ++s) {
        CK(cudaMemcpy(h->geo[s].band_map, em.data(), N * sizeof(int), cudaMemcpyHostToDevice));
        if (h->geo[s].band_bits) CK(cudaMemset(h->geo[s].band_bits, 0, band_bits_words(d) * sizeof(unsigned)));
        CK(cudaMemset(h->geo[s].band_n, 0, 2 * sizeof(int)));
        h->pending[s] = false;
    }
    h->gset = 0;
    h->last_gset = 0;
    CK(cudaMemset(d.sum_row, 0, sizeof(double) * h->row_len));
    CK(cudaMemset(d.sample_count, 0, sizeof(int)));
    CK(cudaMemset(d.status, 0, sizeof(int)));
    CK(cudaMemset(d.rel_pos, 0, sizeof(double) * std::max(1, d.wing_count)));
    long long one = 1;
    CK(cudaMemcpy(d.cycle, &one, sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(d.gcycle, &one, sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemset(d.fin_count, 0, sizeof(int)));
    CK(cudaMemset(d.solve_count, 0, sizeof(int)));
    h->d.movenum = 0;
    h->fields_valid = false;
    h->err_valid = false;
    h->next_cycle = 1;
    h->geo_ready = -1;
    CK(cudaDeviceSynchronize());
    return 0;
}

int ensure_rows(LbmHandle* h, int64_t n) {
    DeviceLock lock(g_device_mutex);
    if (n <= h->rows_cap) return 0;
    if (h->d_rowbuf) {
        cudaFree(h->d_rowbuf);
        h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->d_rowbuf), h->allocs.end());
        h->dev_bytes -= (int64_t)h->rows_cap * h->row_len * sizeof(double);
    }
    int cap = (int)std::max<int64_t>(n, 1024);
    if (dalloc(h, &h->d_rowbuf, (size_t)cap * h->row_len)) return -1;
    h->rows_cap = cap;
    h->d.force_rows = h->d_rowbuf;
    drop_graphs(h);
    h->d.force_rows_cap = cap;
    return 0;
}

int check_status(LbmHandle* h) {
    int st = 0;
    CK(cudaMemcpy(&st, h->d.status, sizeof(int), cudaMemcpyDeviceToHost));
    h->status_seen |= st;
    const int fatal = ST_BAND_OVERFLOW | ST_BOX_OUTSIDE | ST_MOTION | ST_COPY_TIMEOUT | ST_COUPLED_NOCONV;
    if (st & fatal) {
        std::string m = "immersed boundary:";
        if (st & ST_BAND_OVERFLOW) m += " band capacity exceeded;";
        if (st & ST_COUPLED_NOCONV)
            m += " the joint solve of wings whose supports share lattice nodes did not reach its tolerance;";
        if (st & ST_BOX_OUTSIDE) m += " a wing's support box left the lattice;";
        if (st & ST_MOTION) m += " no motion rows loaded;";
        if (st & ST_COPY_TIMEOUT) m += " a shared-memory bulk copy timed out;";
        return fail(h, m);
    }
    return 0;
}

// Event marks around one phase when the phase timers are on.
size_t next_event(LbmHandle* h) {
    if (h->evused == h->evpool.size()) {
        cudaEvent_t e;
        cudaEventCreate(&e);
        h->evpool.push_back(e);
    }
    return h->evused++;
}
struct PhaseMark {
    LbmHandle* h;
    int phase;
    cudaStream_t st;
    size_t a = 0;
    PhaseMark(LbmHandle* h_, int p, cudaStream_t s) : h(h_), phase(p), st(s) {
        if (h->timing) { a = next_event(h); cudaEventRecord(h->evpool[a], st); }
    }
    ~PhaseMark() {
        if (!h->timing) return;
        size_t b = next_event(h);
        cudaEventRecord(h->evpool[b], st);
        h->marks.push_back({phase, {a, b}});
    }
};

void collect_phase_times(LbmHandle* h) {
    for (auto& m : h->marks) {
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, h->evpool[m.second.first], h->evpool[m.second.second]) == cudaSuccess)
            h->phase_ms[m.first] += ms;
    }
    h->marks.clear();
    h->evused = 0;
}

// Fused path: the geometry (motion, markers, band list and factorised G) of
// the first GEO_AHEAD steps of a call, each in its own set; every later
// step's geometry is built GEO_AHEAD steps ahead while earlier steps run.
// The builds run on the side streams (each band list after the previous
// one, the factorisations beside them); the first step or pass waits for
// them.
void build_geometry(LbmHandle* h, int sn, int k);
void prime_geometry(LbmHandle* h) {
    for (bool& p : h->pending) p = false;
    cudaEventRecord(h->ev_main, h->s_main);
    for (int a = 0; a < GEO_AHEAD; ++a) build_geometry(h, (h->gset + a) % GEO_SETS, a & 1);
}

// Makes the main stream wait for every geometry set still building.
void wait_pending(LbmHandle* h) {
    for (int s = 0; s < GEO_SETS; ++s)
        if (h->pending[s]) {
            cudaStreamWaitEvent(h->s_main, h->ev_list[s], 0);
            cudaStreamWaitEvent(h->s_main, h->ev_fact[s], 0);
            h->pending[s] = false;
        }
}

// The geometry of set sn on the side streams (pair k), GEO_AHEAD steps ahead
// of the step that starts it; its band list and factor events let later
// steps wait for it.  Builds read and advance the geometry's cycle counter,
// so a build starts after the previous build's band list.
void build_geometry(LbmHandle* h, int sn, int k) {
    DevState dn = h->d;
    use_geo(dn, h->geo[sn]);
    cudaStream_t sa = h->s_aux[k], sb = h->s_aux2[k];
    cudaStreamWaitEvent(sa, h->ev_main, 0);
    const int sp = (sn + GEO_SETS - 1) % GEO_SETS;
    if (h->pending[sp]) cudaStreamWaitEvent(sa, h->ev_list[sp], 0);
    {
        PhaseMark pm(h, 0, sa);
        launch_ibm_band(dn, sa, h->ev_geom[sn]);
    }
    cudaEventRecord(h->ev_list[sn], sa);
    cudaStreamWaitEvent(sb, h->ev_geom[sn], 0);
    {
        PhaseMark pm(h, 5, sb);
        launch_ibm_factor(dn, h->factor_smem, sb);
    }
    cudaEventRecord(h->ev_fact[sn], sb);
    h->pending[sn] = true;
}

// One evolution step (solution.f90:272-422) on the current planes.  On the
// fused path, prefetch builds the geometry of the step GEO_AHEAD ahead, and
// drain makes this step wait for it as well (graph boundaries).
void enqueue_step(LbmHandle* h, bool fields, bool diag, bool prefetch, bool drain) {
    DevState d = current(h);
    d.diag = diag ? 1 : 0;
    d.write_fields = fields ? 1 : 0;
    if (d.precision == 0) {
        {
            PhaseMark pm(h, 0, h->s_main);
            launch_ibm_band(d, h->s_main, nullptr);    // mode + move_boundary (:292-299)
        }
        {
            PhaseMark pm(h, 1, h->s_main);
            launch_plain_stream(d, h->s_main);         // streaming (:318)
            launch_plain_moments(d, h->s_main);        // physical_variables (:321)
        }
        {
            PhaseMark pm(h, 5, h->s_main);             // immersed_boundary_wu (:325)
            launch_ibm_factor(d, h->factor_smem, h->s_main);
        }
        {
            PhaseMark pm(h, 4, h->s_main);
            launch_ibm_rhs(d, false, h->s_main);
            launch_ibm_solve(d, false, false, h->s_main);
        }
        {
            PhaseMark pm(h, 1, h->s_main);
            launch_plain_collide(d, h->s_main);        // colission (:328)
        }
        {
            PhaseMark pm(h, 3, h->s_main);
            launch_outer_bc(d, h->s_main);             // boundary_condition1 (:420)
        }
        launch_step_advance(d, h->s_main);
    } else {
        // The immersed boundary, the far field and a later step's geometry
        // overlap the bulk kernel.  All read only the current planes, and the
        // writes go to disjoint nodes of the next planes (interior, band,
        // border).  Support boxes keep off the border rows and columns the far
        // field reads, so it needs nothing from the immersed boundary.  The
        // geometry of this step was built GEO_AHEAD steps ago (or by the
        // prime); the one built now goes to the set whose last reader was
        // the previous step.
        const int sn = (h->gset + GEO_AHEAD) % GEO_SETS, s1 = (h->gset + 1) % GEO_SETS;
        if (h->pending[h->gset]) {   // this step's geometry, primed on the side streams
            cudaStreamWaitEvent(h->s_main, h->ev_list[h->gset], 0);
            cudaStreamWaitEvent(h->s_main, h->ev_fact[h->gset], 0);
            h->pending[h->gset] = false;
        }
        cudaEventRecord(h->ev_main, h->s_main);
        cudaStreamWaitEvent(h->s_ibm, h->ev_main, 0);
        cudaStreamWaitEvent(h->s_bc, h->ev_main, 0);
        if (prefetch) build_geometry(h, sn, h->gset & 1);
        {
            PhaseMark pm(h, 3, h->s_bc);
            launch_outer_bc(d, h->s_bc);
        }
        cudaEventRecord(h->ev_bc, h->s_bc);
        {
            // rhs, substitution, spread, then one closing kernel: band nodes
            // re-collided (the bulk kernel leaves them out), force row, cycle
            // advance
            PhaseMark pm(h, 4, h->s_ibm);
            launch_ibm_rhs(d, true, h->s_ibm);
            launch_ibm_solve(d, true, fields, h->s_ibm);
        }
        cudaEventRecord(h->ev_ibm, h->s_ibm);
        {
            PhaseMark pm(h, 1, h->s_main);
            launch_fused_bulk(d, h->fc, fields, h->tmap_ok ? &h->tmap[h->cur] : nullptr, h->s_main);
        }
        cudaStreamWaitEvent(h->s_main, h->ev_ibm, 0);
        cudaStreamWaitEvent(h->s_main, h->ev_bc, 0);
        // the next step starts once its geometry is complete
        for (int s : {s1, sn}) {
            if (!h->pending[s] || (s != s1 && !drain)) continue;
            cudaStreamWaitEvent(h->s_main, h->ev_list[s], 0);
            cudaStreamWaitEvent(h->s_main, h->ev_fact[s], 0);
            h->pending[s] = false;
        }
        h->cur = third_planes(h);
        h->last_gset = h->gset;
        h->gset = s1;
    }
    if (h->timing) h->timed_steps += 1;
}

// Two steps n -> n + 2 of the fused path in one pass (no fields, no
// diagnostics): P = planes[cur] (step n), O = planes[alt] (step n + 1 where
// the second step's immersed boundary and far field and the near tiles read
// it), Q = the third copy (step n + 2).
//   s_ibm   chain of step n (P -> O at its band nodes), then, after the
//           ring, the chain of step n + 1 (O -> Q at its band nodes)
//   s_bc    far field of step n (P -> O border), the ring (P -> O: the
//           support boxes of step n + 1 and one ring around them, the
//           columns and rows the far field reads), then, after the first
//           chain (a band node may sit in column 3), the far field of
//           step n + 1 (O -> Q border)
//   s_main  far tiles (P -> Q), once the first chain's rhs is done
//   s_near  near tiles (P and O -> Q), after the first chain and far field
//   aux     the geometry of steps n + 2 and n + 3
// The pass ends when all are done (the next pass reads all of them).
// diag_last: the pass ends the call, so its second step computes the
// no-slip residual diagnostic (lbm_ibm_residual).
void enqueue_pass(LbmHandle* h, bool diag_last = false) {
    wait_pending(h);   // both steps' geometry is complete before the pass starts
    const int g0 = h->gset, g1 = (g0 + 1) % GEO_SETS, g2 = (g0 + 2) % GEO_SETS, g3 = (g0 + 3) % GEO_SETS;
    const int third = third_planes(h);
    float *P = h->planes[h->cur], *O = h->planes[h->alt], *Q = h->planes[third];
    DevState dA = h->d, dB = h->d;
    dA.diag = 0;
    dB.diag = diag_last ? 1 : 0;
    dA.write_fields = dB.write_fields = 0;
    dA.gA = P;
    dA.gB = O;
    use_geo(dA, h->geo[g0]);
    dB.gA = O;
    dB.gB = Q;
    use_geo(dB, h->geo[g1]);
    PassArgs pa;
    pa.P = P;
    pa.O = O;
    pa.Q = Q;
    pa.bits0 = h->geo[g0].band_bits;
    pa.bits1 = h->geo[g1].band_bits;
    pa.flags0 = h->geo[g0].tile_flags;
    pa.border_list = h->border_tiles;
    pa.band_list = h->geo[g0].tile_list;
    pa.band_n = h->geo[g0].tile_n;
    pa.nborder = h->nborder;
    pa.band_cap = std::min(h->d.pass_ntx * h->d.pass_nty,
                           pass_tiles_per_segment(h->d.pass_rows) * std::max(1, h->d.nseg));
    pa.nx = h->d.nx;
    pa.ny = h->d.ny;
    pa.pitch = h->d.pitch;
    pa.ntx = h->d.pass_ntx;
    pa.nty = h->d.pass_nty;
    pa.rows = h->d.pass_rows;
    pa.plane = h->d.plane;
    pa.c = h->fc;
    pa.k = pass_pairs(h->fc);
    pa.status = h->d.status;
    pa.far_tiles = h->timing ? h->d_far_tiles : nullptr;
    cudaEventRecord(h->ev_main, h->s_main);
    for (cudaStream_t st : {h->s_ibm, h->s_bc, h->s_near}) cudaStreamWaitEvent(st, h->ev_main, 0);
    build_geometry(h, g2, 0);
    build_geometry(h, g3, 1);
    {
        PhaseMark pm(h, 3, h->s_bc);
        launch_outer_bc(dA, h->s_bc);
    }
    cudaEventRecord(h->ev_bc1, h->s_bc);
    {
        PhaseMark pm(h, 2, h->s_bc);
        launch_pass_ring(dB, P, O, pa.bits0, h->s_bc);
    }
    cudaEventRecord(h->ev_ring, h->s_bc);
    {
        PhaseMark pm(h, 4, h->s_ibm);
        launch_ibm_rhs(dA, true, h->s_ibm);
        // the far tiles start once the first rhs is done: the substitution
        // block then finds an SM before the far tiles fill them all (its
        // shared memory can exceed what one far-tile block frees, and
        // lower-priority blocks that fit are placed first)
        cudaEventRecord(h->ev_rhs1, h->s_ibm);
        cudaStreamWaitEvent(h->s_main, h->ev_rhs1, 0);
        launch_ibm_solve(dA, true, false, h->s_ibm, true);
    }
    cudaEventRecord(h->ev_chain1, h->s_ibm);
    cudaStreamWaitEvent(h->s_ibm, h->ev_ring, 0);
    {
        PhaseMark pm(h, 4, h->s_ibm);
        launch_ibm_rhs(dB, true, h->s_ibm);
        launch_ibm_solve(dB, true, false, h->s_ibm, true);
    }
    cudaEventRecord(h->ev_ibm, h->s_ibm);
    cudaStreamWaitEvent(h->s_bc, h->ev_chain1, 0);
    {
        PhaseMark pm(h, 3, h->s_bc);
        launch_outer_bc(dB, h->s_bc);
    }
    cudaEventRecord(h->ev_bc, h->s_bc);
    cudaStreamWaitEvent(h->s_near, h->ev_chain1, 0);
    cudaStreamWaitEvent(h->s_near, h->ev_bc1, 0);
    {
        PhaseMark pm(h, 2, h->s_near);
        launch_pass_near(pa, &h->ptmap[h->cur], h->s_near);
    }
    cudaEventRecord(h->ev_near, h->s_near);
    {
        PhaseMark pm(h, 1, h->s_main), pf(h, 6, h->s_main);
        launch_pass_far(pa, &h->ptmap[h->cur], h->s_main);
    }
    for (cudaEvent_t e : {h->ev_ibm, h->ev_bc, h->ev_near, h->ev_list[g2], h->ev_fact[g2], h->ev_list[g3],
                          h->ev_fact[g3]})
        cudaStreamWaitEvent(h->s_main, e, 0);
    for (bool& q : h->pending) q = false;
    h->cur = third;   // O stays the overlay of the next pass; P is free
    h->last_gset = g1;
    h->gset = g2;
    if (h->timing) {
        h->timed_steps += 2;
        h->timed_passes += 1;
    }
}

void drop_graphs(LbmHandle* h) {
    for (auto* tab : {&h->gexec, &h->pexec})
        for (auto& plane : *tab)
            for (auto& row : plane)
                for (auto& g : row)
                    if (g) {
                        cudaGraphExecDestroy(g);
                        g = nullptr;
                    }
}

// GRAPH_STEPS single steps, or one pass, from planes (c, a) and geometry
// set gs, captured from all streams (the side streams join and leave
// through events, as in eager launches).  The graph is self-contained: it
// starts with the geometry of its first GEO_AHEAD steps complete and its
// last step waits for the geometry it built for the steps after the graph.
int build_graph(LbmHandle* h, int c, int a, int gs, bool pass) {
    DeviceLock lock(g_device_mutex);
    // the capture re-records the geometry events: wait for pending builds
    // now, while the events still name them
    wait_pending(h);
    const int saved_c = h->cur, saved_a = h->alt, saved_g = h->gset, saved_last = h->last_gset;
    bool saved_pending[GEO_SETS];
    std::copy(h->pending, h->pending + GEO_SETS, saved_pending);
    h->cur = c;
    h->alt = a;
    h->gset = gs;
    for (bool& q : h->pending) q = false;
    cudaGraph_t g = nullptr;
    CK(cudaStreamBeginCapture(h->s_main, cudaStreamCaptureModeThreadLocal));
    if (pass)
        enqueue_pass(h);
    else
        for (int k = 0; k < GRAPH_STEPS; ++k) enqueue_step(h, false, false, true, k == GRAPH_STEPS - 1);
    cudaError_t e = cudaStreamEndCapture(h->s_main, &g);
    h->cur = saved_c;
    h->alt = saved_a;
    h->gset = saved_g;
    h->last_gset = saved_last;
    std::copy(saved_pending, saved_pending + GEO_SETS, h->pending);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaStreamEndCapture");
    // Graph launches run every node at the priority of the launch stream
    // unless nodes carry their own: the bulk kernel gets the low priority,
    // the far field and the geometry kernels the middle one and the
    // immersed-boundary chain the high one, so all are dispatched ahead of
    // pending bulk blocks instead of after the bulk grid, the chain first.
    size_t nn = 0;
    e = cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g, nodes.data(), &nn);
    for (size_t k = 0; e == cudaSuccess && k < nn; ++k) {
        cudaGraphNodeType ty;
        e = cudaGraphNodeGetType(nodes[k], &ty);
        if (e != cudaSuccess || ty != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        e = cudaGraphKernelNodeGetParams(nodes[k], &kp);
        if (e != cudaSuccess) break;
        cudaKernelNodeAttrValue v;
        std::memset(&v, 0, sizeof(v));
        v.priority = (is_bulk_kernel(kp.func) || is_pass_far_kernel(kp.func)) ? h->prio_lo
                     : (is_geometry_kernel(kp.func) || is_far_field_kernel(kp.func) || is_pass_near_kernel(kp.func))
                         ? h->prio_mid
                         : h->prio_hi;
        e = cudaGraphKernelNodeSetAttribute(nodes[k], cudaKernelNodeAttributePriority, &v);
    }
    cudaGraphExec_t& slot = pass ? h->pexec[c][a][gs] : h->gexec[c][a][gs];
    if (e == cudaSuccess) e = cudaGraphInstantiate(&slot, g, cudaGraphInstantiateFlagUseNodePriority);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(h, e, "cudaGraphInstantiate");
    return 0;
}

void drop_batch_graphs(LbmBatch* b) {
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

// A graph's kernel nodes run at the priority of the launch stream unless
// they carry their own: bulk low; far field, geometry and factorisation
// middle; the immersed-boundary chain high, as the batch's streams have.
cudaError_t instantiate_with_priorities(LbmBatch* b, cudaGraph_t g, cudaGraphExec_t* out) {
    size_t nn = 0;
    cudaError_t e = cudaGraphGetNodes(g, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (e == cudaSuccess && nn) e = cudaGraphGetNodes(g, nodes.data(), &nn);
    for (size_t k = 0; e == cudaSuccess && k < nn; ++k) {
        cudaGraphNodeType ty;
        e = cudaGraphNodeGetType(nodes[k], &ty);
        if (e != cudaSuccess || ty != cudaGraphNodeTypeKernel) continue;
        cudaKernelNodeParams kp;
        e = cudaGraphKernelNodeGetParams(nodes[k], &kp);
        if (e != cudaSuccess) break;
        cudaKernelNodeAttrValue v;
        std::memset(&v, 0, sizeof(v));
        v.priority = is_bulk_multi_kernel(kp.func) ? b->prio_lo
                     : (is_far_field_multi_kernel(kp.func) || is_geometry_multi_kernel(kp.func)) ? b->prio_mid
                                                                                                 : b->prio_hi;
        e = cudaGraphKernelNodeSetAttribute(nodes[k], cudaKernelNodeAttributePriority, &v);
    }
    if (e == cudaSuccess) e = cudaGraphInstantiate(out, g, cudaGraphInstantiateFlagUseNodePriority);
    return e;
}

int batch_fail(LbmBatch* b, const std::string& msg) {
    if (b) b->err = msg;
    return -1;
}

#define BCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess) return batch_fail(b, std::string("CUDA error in ") + #call + ": " +  \
                                                         cudaGetErrorString(e_));                    \
    } while (0)

int multi_blocks(MultiKernel k, const DevState& d) {
    int n = multi_blocks_ibm(k, d);
    if (n < 0) n = multi_blocks_solver(k, d);
    if (n < 0) n = multi_blocks_fused(k, d);
    return std::max(n, 0);
}

// Per handle of a batch, eight states: the plain step, the second-last and
// the last step of the call (the field and diagnostic flags of lbm_step),
// and the geometry built one step ahead, each for the two plane parities /
// geometry sets a step can start from.
constexpr int BV_PLAIN = 0, BV_SECOND_LAST = 2, BV_LAST = 4, BV_AHEAD = 6, BV_COUNT = 8;
constexpr int BATCH_SLOT_ITEMS = 4;   // per-slot items per thread in packed launches
constexpr int64_t GRAPH_PAIR_MIN = 8;  // steady steps ahead before a step pair is captured

// Packed steps alternate between the handle's current plane copy and its
// third copy (as single steps do) and between two of its geometry sets
// (gset, gset + 1), each step building the next step's geometry into the
// other set.
int batch_set(const LbmHandle* h, int ph) { return (h->gset + (ph & 1)) % GEO_SETS; }

void batch_variants(LbmHandle* h, bool want_fields, bool want_err, DevState* out) {
    for (int ph = 0; ph < 2; ++ph) {
        DevState d = h->d;
        const int g = batch_set(h, ph);
        const int third = third_planes(h);
        d.gA = h->planes[ph ? third : h->cur];
        d.gB = h->planes[ph ? h->cur : third];
        use_geo(d, h->geo[g]);
        d.tile_flags = nullptr;   // no passes in packed steps
        d.diag = 0;
        d.write_fields = 0;
        d.slot_items = BATCH_SLOT_ITEMS;
        out[BV_PLAIN + ph] = d;
        DevState sl = d;
        sl.write_fields = want_err ? 1 : 0;
        out[BV_SECOND_LAST + ph] = sl;
        DevState l = d;
        l.write_fields = (want_fields || want_err) ? 1 : 0;
        l.diag = 1;
        if (want_err) {   // the previous step's velocity becomes u0
            std::swap(l.fo_u, l.fo_u0);
            std::swap(l.fo_v, l.fo_v0);
        }
        out[BV_LAST + ph] = l;
        DevState a = d;
        use_geo(a, h->geo[batch_set(h, ph + 1)]);
        a.tile_flags = nullptr;
        out[BV_AHEAD + ph] = a;
    }
}

int copy_pitched_out(LbmHandle* h, const double* src, double* dst) {
    const DevState& d = h->d;
    CK(cudaMemcpy2D(dst, sizeof(double) * d.nx, src, sizeof(double) * d.pitch, sizeof(double) * d.nx, d.ny,
                    cudaMemcpyDeviceToHost));
    return 0;
}

}  // namespace

extern "C" {

int lbm_abi_version(void) { return LBM_ABI_VERSION; }

void lbm_config_default(LbmConfig* c) {
    std::memset(c, 0, sizeof(*c));
    c->nx = 4001; c->ny = 2001; c->scale = 0.01; c->uu = 0.01; c->re = 500.0;
    c->ox = -20.0; c->oy = -10.0;
    const double s[9] = {0.0, 1.1, 1.05, 0.0, 1.2, 0.0, 1.2, 0.0, 0.0};
    for (int k = 0; k < 9; ++k) c->s[k] = s[k];
    c->wing_count = 2; c->wing_x_origin = 0.0; c->wing_x_spacing = 1.5; c->wing_y_origin = 0.5;
    c->motion_source = LBM_MOTION_FILE; c->precision = LBM_PRECISION_FP64; c->device = 0;
}

int lbm_create(const LbmConfig* cfg, const double* markers_xy, const int32_t* points_per_wing, LbmHandle** out) {
    DeviceLock lock(g_device_mutex);
    if (!out) return -1;
    *out = nullptr;
    LbmHandle* h = new LbmHandle();
    *out = h;
    if (!cfg) return fail(h, "null config");
    h->cfg = *cfg;
    const LbmConfig& c = *cfg;
    if (c.nx < 6 || c.ny < 6) return fail(h, "lattice must be at least 6 x 6 nodes");
    if (!(c.scale > 0.0) || !(c.uu > 0.0) || !(c.re > 0.0)) return fail(h, "scale, uu and re must be positive");
    if (c.wing_count < 0 || c.wing_count > 16) return fail(h, "wing_count must be in [0, 16]");
    if (c.precision != LBM_PRECISION_FP64 && c.precision != LBM_PRECISION_FP32)
        return fail(h, "unknown precision");
    if (c.motion_source != LBM_MOTION_FILE && c.motion_source != LBM_MOTION_STREAM)
        return fail(h, "unknown motion source");
    if (c.precision == LBM_PRECISION_FP32 && (c.s[0] != 0.0 || c.s[3] != 0.0 || c.s[5] != 0.0))
        return fail(h, "the fused path relaxes only the non-conserved moments (s[0], s[3], s[5] must be 0)");
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    if (c.device < 0 || c.device >= ndev) return fail(h, "CUDA device not available");
    CK(cudaSetDevice(c.device));

    DevState& d = h->d;
    d.nx = c.nx; d.ny = c.ny;
    d.pitch = (c.nx + 31) / 32 * 32;
    d.plane = (long long)d.pitch * c.ny;
    d.scale = c.scale; d.uu = c.uu; d.ox = c.ox; d.oy = c.oy;
    // ini_mesh.f90:30-31, 59-67
    const double niu = c.uu * (1.0 / c.scale) / c.re;
    const double tau = 3.0 * niu + 0.5;
    for (int k = 0; k < 9; ++k) d.s[k] = c.s[k];
    if (d.s[7] <= 0.0) d.s[7] = 1.0 / tau;
    if (d.s[8] <= 0.0) d.s[8] = 1.0 / tau;
    gauss_jordan_inverse(d.minv);
    d.precision = c.precision;
    d.wing_count = c.wing_count;
    d.wing_x_origin = c.wing_x_origin; d.wing_x_spacing = c.wing_x_spacing; d.wing_y_origin = c.wing_y_origin;
    d.xc = c.xc; d.yc = c.yc;
    d.motion_source = c.motion_source;
    d.ncol = 1 + 9 * c.wing_count;
    h->row_len = 4 + 12 * c.wing_count;

    // geometry (airfoil.f90:207-242)
    const int W = c.wing_count;
    std::vector<int> pstart(W), sstart(W), npts(W), segw;
    int np = 0, ns = 0;
    for (int w = 0; w < W; ++w) {
        if (!points_per_wing || points_per_wing[w] < 3) return fail(h, "each wing needs at least 3 points");
        pstart[w] = np; sstart[w] = ns; npts[w] = points_per_wing[w];
        np += points_per_wing[w];
        ns += points_per_wing[w] - 1;
        for (int k = 0; k < points_per_wing[w] - 1; ++k) segw.push_back(w);
    }
    if (W > 0 && !markers_xy) return fail(h, "markers_xy is null");
    d.npts = np; d.nseg = ns;
    h->xb0.resize(np); h->yb0.resize(np);
    for (int p = 0; p < np; ++p) {
        h->xb0[p] = markers_xy[2 * p] + (c.xc - 0.0);
        h->yb0[p] = markers_xy[2 * p + 1] + (c.yc - 0.0);
    }
    // RCM order and half bandwidth per wing
    std::vector<int> perm(ns), bw(W), rpos(ns);
    std::vector<long long> lofs(W), iofs(W), qofs(W);
    long long ltot = 0, itot = 0, qtot = 0, qmax = 0;
    for (int w = 0; w < W; ++w) {
        const int nw = npts[w] - 1;
        std::vector<double> mx(nw), my(nw);
        for (int k = 0; k < nw; ++k) {
            int p = pstart[w] + k;
            mx[k] = 0.5 * (h->xb0[p + 1] + h->xb0[p]);
            my[k] = 0.5 * (h->yb0[p + 1] + h->yb0[p]);
        }
        std::vector<int> ord;
        bw[w] = rcm_order(mx, my, c.scale, ord);
        for (int k = 0; k < nw; ++k) {
            perm[sstart[w] + k] = sstart[w] + ord[k];
            rpos[sstart[w] + ord[k]] = k;
        }
        lofs[w] = ltot;   // start of the wing's storage (its leading zero row)
        ltot += ibm_wing_storage(nw, bw[w]);
        iofs[w] = itot;
        itot += ibm_linv_storage(nw);
        qofs[w] = qtot;   // the wing's 32-row panel data
        qtot += ibm_panel32_storage(nw, bw[w]);
        qmax = std::max(qmax, ibm_panel32_storage(nw, bw[w]));
    }

    // allocations
    const size_t N = (size_t)d.plane;
    if (c.precision == LBM_PRECISION_FP64) {
        if (dalloc(h, &d.f, 9 * N) || dalloc(h, &d.f0, 9 * N) || dalloc(h, &d.rho, N) || dalloc(h, &d.u, N) ||
            dalloc(h, &d.v, N) || dalloc(h, &d.u0, N) || dalloc(h, &d.v0, N) || dalloc(h, &d.pre, N) ||
            dalloc(h, &d.gfx, N) || dalloc(h, &d.gfy, N))
            return -1;
    } else {
        if (dalloc(h, &h->planes[0], 9 * N) || dalloc(h, &h->planes[1], 9 * N) ||
            dalloc(h, &h->planes[2], 9 * N) || dalloc(h, &d.edge_f0, 9 * (size_t)(2 * c.nx + 2 * c.ny)))
            return -1;
    }
    if (dalloc(h, &d.band_map, N)) return -1;
    if (c.precision != LBM_PRECISION_FP64 && dalloc(h, &d.band_bits, band_bits_words(d))) return -1;
    d.band_cap = std::max(64, BOX_SLOTS * ns);
    d.slot_items = 1;
    const int cap = d.band_cap;
    int* band_n = nullptr;
    if (dalloc(h, &band_n, 2) || dalloc(h, &d.band_ij, 2 * (size_t)cap) || dalloc(h, &d.band_wing, cap) ||
        dalloc(h, &d.band_rho, cap) || dalloc(h, &d.band_us, cap) || dalloc(h, &d.band_vs, cap) ||
        dalloc(h, &d.band_du, cap) || dalloc(h, &d.band_dv, cap) )
        return -1;
    d.band_n = band_n;
    int *pst = nullptr, *sst = nullptr, *npw = nullptr, *sgw = nullptr, *dperm = nullptr, *dbw = nullptr,
        *drpos = nullptr;
    long long *dlofs = nullptr, *diofs = nullptr, *dqofs = nullptr;
    double *xb0 = nullptr, *yb0 = nullptr;
    const size_t nsz = std::max(1, ns), npz = std::max(1, np), wz = std::max(1, W);
    if (dalloc(h, &pst, wz) || dalloc(h, &sst, wz) || dalloc(h, &npw, wz) || dalloc(h, &sgw, nsz) ||
        dalloc(h, &xb0, npz) || dalloc(h, &yb0, npz) || dalloc(h, &d.xb1, npz) || dalloc(h, &d.yb1, npz) ||
        dalloc(h, &d.xb2, nsz) || dalloc(h, &d.yb2, nsz) || dalloc(h, &d.box, 4 * nsz) ||
        dalloc(h, &d.claim_cnt, nsz + 1) || dalloc(h, &d.kx, 6 * nsz) || dalloc(h, &d.ky, 6 * nsz) ||
        dalloc(h, &d.pb, nsz * BOX_SLOTS) || dalloc(h, &drpos, nsz) || dalloc(h, &d.band_claimer, (size_t)cap) ||
        dalloc(h, &d.rx, nsz) || dalloc(h, &d.ry, nsz) || dalloc(h, &d.qx, nsz) || dalloc(h, &d.qy, nsz) ||
        dalloc(h, &d.cg_work, 8 * nsz) || dalloc(h, &d.solve_count, 1) ||
        dalloc(h, &dperm, nsz) || dalloc(h, &dbw, wz) || dalloc(h, &dlofs, wz) ||
        dalloc(h, &d.lband, (size_t)std::max<long long>(1, ltot)) || dalloc(h, &diofs, wz) ||
        dalloc(h, &d.linv, (size_t)std::max<long long>(1, itot)) || dalloc(h, &d.wm, wz) ||
        dalloc(h, &d.lq, (size_t)std::max<long long>(1, qtot)) || dalloc(h, &dqofs, wz) ||
        dalloc(h, &d.rel_pos, wz) || dalloc(h, &d.cycle, 1) || dalloc(h, &d.row_index, 1) ||
        dalloc(h, &d.gcycle, 1) || dalloc(h, &d.fin_count, 1) ||
        dalloc(h, &d.sum_row, (size_t)h->row_len) || dalloc(h, &d.sample_count, 1) || dalloc(h, &d.status, 1) ||
        dalloc(h, &d.wing_fm, 3 * wz) || dalloc(h, &d.ibm_resid, 2) || dalloc(h, &d.stream_start, (size_t)d.ncol) ||
        dalloc(h, &d.stream_target, (size_t)d.ncol))
        return -1;
    if (dalloc(h, &h->err_partial, 2 * (size_t)err_partial_count()) || dalloc(h, &h->err_out, 1)) return -1;
    if (W > 0) {
        CK(cudaMemcpy(pst, pstart.data(), W * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(sst, sstart.data(), W * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(npw, npts.data(), W * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(sgw, segw.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(xb0, h->xb0.data(), np * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(yb0, h->yb0.data(), np * sizeof(double), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dperm, perm.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(drpos, rpos.data(), ns * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dbw, bw.data(), W * sizeof(int), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dlofs, lofs.data(), W * sizeof(long long), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(diofs, iofs.data(), W * sizeof(long long), cudaMemcpyHostToDevice));
        CK(cudaMemcpy(dqofs, qofs.data(), W * sizeof(long long), cudaMemcpyHostToDevice));
    }
    d.wing_pstart = pst; d.wing_sstart = sst; d.wing_npts = npw; d.seg_wing = sgw;
    d.xb0 = xb0; d.yb0 = yb0; d.perm = dperm; d.wing_bw = dbw; d.wing_lofs = dlofs; d.rpos = drpos;
    d.wing_linv_ofs = diofs;
    d.wing_qofs = dqofs;
    d.q32_doubles_max = qmax;
    h->ppw.assign(npts.begin(), npts.end());
    // dynamic shared memory of the factorisation kernel (one block per wing):
    // [staged panel rows][pair table][the wing's banded factor, if it fits]
    int bwmax = 1, nwmax = 1;
    long long wmax = 0;
    for (int w = 0; w < W; ++w) {
        bwmax = std::max(bwmax, bw[w]);
        nwmax = std::max(nwmax, npts[w] - 1);
        wmax = std::max<long long>(wmax, ibm_wing_storage(npts[w] - 1, bw[w]));
    }
    if (bwmax > IBM_MAX_BANDWIDTH)
        return fail(h, "immersed boundary: markers too dense for the banded solver (half bandwidth " +
                           std::to_string(bwmax) + " > " + std::to_string(IBM_MAX_BANDWIDTH) + ")");
    d.bw_max = bwmax;
    d.nw_max = nwmax;
    d.lband_total = ltot;
    const size_t base = ibm_factor_staging_bytes(bwmax);
    const size_t smem_cap = 200 * 1024;
    d.factor_smem_off = (long long)base;
    d.factor_in_smem = base + (size_t)wmax * sizeof(double) <= smem_cap ? 1 : 0;
    h->factor_smem = d.factor_in_smem ? base + (size_t)wmax * sizeof(double) : base;
    if (h->factor_smem > smem_cap) return fail(h, "immersed boundary: too many segments for one factorisation block");
    // substitution: the wing's factor goes to shared memory when it fits
    if (ibm_solve_smem(nwmax, bwmax, wmax, false) > smem_cap)
        return fail(h, "immersed boundary: too many segments for one substitution block");
    d.solve_in_smem = ibm_solve_smem(nwmax, bwmax, wmax, true) <= smem_cap && !(c.flags & LBM_FLAG_SOLVE_STREAM);
    d.solve_smem = (long long)ibm_solve_smem(nwmax, bwmax, wmax, d.solve_in_smem != 0);
    // else a ring of factor rows when it fits (wings of many markers)
    d.solve_stream = !d.solve_in_smem && ibm_solve_ring_fits(bwmax) &&
                     ibm_solve_smem(nwmax, bwmax, wmax, false) + ibm_solve_ring_bytes(bwmax) <= smem_cap;
    if (d.solve_stream) d.solve_smem += (long long)ibm_solve_ring_bytes(bwmax);
    // substitution in 32-row panels on request, when every wing's panel
    // data fit in shared memory (the factorisation then also builds them)
    d.solve32 = (c.flags & LBM_FLAG_SOLVE_PANELS32) && W > 0 && !(c.flags & LBM_FLAG_SOLVE_STREAM) &&
                ibm_solve32_smem(qmax, nwmax, bwmax) <= smem_cap;
    if (d.solve32) d.solve_smem = (long long)ibm_solve32_smem(qmax, nwmax, bwmax);
    CK(ibm_prepare(h->factor_smem, (size_t)d.solve_smem));
    if (dalloc(h, &d.piv_floor, wz) || dalloc(h, &d.ymax, 2 * wz) || dalloc(h, &d.ibm_flags, 4) ||
        dalloc(h, &d.force_part, (size_t)ibm_finish_blocks(d) * wz * 3))
        return -1;
    // the second geometry set (fused path: the next step's geometry)
    h->geo[0] = geo_of(d);
    for (int s = 1; s < GEO_SETS; ++s) h->geo[s] = h->geo[0];
    for (int s = 1; s < GEO_SETS && c.precision != LBM_PRECISION_FP64; ++s) {
        GeoSet& g = h->geo[s];
        if (dalloc(h, &g.wm, wz) || dalloc(h, &g.xb1, npz) || dalloc(h, &g.yb1, npz) || dalloc(h, &g.xb2, nsz) ||
            dalloc(h, &g.yb2, nsz) || dalloc(h, &g.kx, 6 * nsz) || dalloc(h, &g.ky, 6 * nsz) ||
            dalloc(h, &g.box, 4 * nsz) || dalloc(h, &g.claim_cnt, nsz + 1) || dalloc(h, &g.pb, nsz * BOX_SLOTS) ||
            dalloc(h, &g.band_claimer, (size_t)cap) || dalloc(h, &g.band_n, 2) ||
            dalloc(h, &g.band_ij, 2 * (size_t)cap) || dalloc(h, &g.band_wing, cap) || dalloc(h, &g.band_map, N) ||
            dalloc(h, &g.band_bits, band_bits_words(d)) ||
            dalloc(h, &g.ibm_flags, 4) || dalloc(h, &g.lband, (size_t)std::max<long long>(1, ltot)) ||
            dalloc(h, &g.linv, (size_t)std::max<long long>(1, itot)) ||
            dalloc(h, &g.lq, (size_t)std::max<long long>(1, qtot)))
            return -1;
    }
    if (c.precision != LBM_PRECISION_FP64) {
        // pass tiles: flags and flagged-tile lists per geometry set, and the
        // tiles whose R1 meets the border; the tall tiles on large lattices
        // (or as the flags ask)
        const bool tall = (c.flags & LBM_FLAG_PASS_TALL_TILES) ||
                          (!(c.flags & LBM_FLAG_PASS_SHORT_TILES) && (long long)c.nx * c.ny >= PASS_TALL_NODES);
        const int rows = tall ? PASS_TY_TALL : PASS_TY;
        const int ntx = pass_tiles_x(c.nx), nty = pass_tiles_y(c.ny, rows), ntl = ntx * nty;
        for (int s = 0; s < GEO_SETS; ++s) {
            GeoSet& g = h->geo[s];
            if (dalloc(h, &g.tile_flags, (size_t)(ntl + 3) / 4 * 4) || dalloc(h, &g.tile_list, (size_t)ntl) ||
                dalloc(h, &g.tile_n, 1))
                return -1;
            CK(cudaMemset(g.tile_flags, 0, (size_t)(ntl + 3) / 4 * 4));
            CK(cudaMemset(g.tile_n, 0, sizeof(int)));
        }
        h->d.tile_flags = h->geo[0].tile_flags;
        h->d.tile_list = h->geo[0].tile_list;
        h->d.tile_n = h->geo[0].tile_n;
        h->d.pass_ntx = ntx;
        h->d.pass_nty = nty;
        h->d.pass_rows = rows;
        std::vector<int> bt;
        for (int t = 0; t < ntl; ++t)
            if (pass_border_tile(t % ntx, t / ntx, c.nx, c.ny, rows)) bt.push_back(t);
        if (dalloc(h, &h->border_tiles, bt.size()) || dalloc(h, &h->d_far_tiles, 1)) return -1;
        CK(cudaMemset(h->d_far_tiles, 0, sizeof(int)));
        CK(cudaMemcpy(h->border_tiles, bt.data(), bt.size() * sizeof(int), cudaMemcpyHostToDevice));
        h->nborder = (int)bt.size();
    }
    if (ensure_rows(h, 1024)) return -1;
    // the immersed-boundary chain is latency-bound and on the critical path:
    // its stream gets the highest priority so its blocks are scheduled ahead
    // of waiting bulk blocks; the far field and the geometry built a step
    // ahead have slack until the step ends and take the middle priority, so
    // they never delay the chain
    int prio_lo = 0, prio_hi = 0;
    CK(cudaDeviceGetStreamPriorityRange(&prio_lo, &prio_hi));
    h->prio_lo = prio_lo;
    h->prio_hi = prio_hi;
    h->prio_mid = (prio_lo + prio_hi) / 2;
    CK(cudaStreamCreateWithPriority(&h->s_main, cudaStreamNonBlocking, prio_lo));
    CK(cudaStreamCreateWithPriority(&h->s_ibm, cudaStreamNonBlocking, prio_hi));
    for (int k = 0; k < 2; ++k) {
        CK(cudaStreamCreateWithPriority(&h->s_aux[k], cudaStreamNonBlocking, h->prio_mid));
        CK(cudaStreamCreateWithPriority(&h->s_aux2[k], cudaStreamNonBlocking, h->prio_mid));
    }
    for (int s = 0; s < GEO_SETS; ++s) CK(cudaEventCreateWithFlags(&h->ev_geom[s], cudaEventDisableTiming));
    CK(cudaStreamCreateWithPriority(&h->s_bc, cudaStreamNonBlocking, h->prio_mid));
    CK(cudaStreamCreateWithPriority(&h->s_near, cudaStreamNonBlocking, h->prio_mid));
    for (cudaEvent_t* e :
         {&h->ev_ibm, &h->ev_main, &h->ev_bc, &h->ev_rhs1, &h->ev_chain1, &h->ev_bc1, &h->ev_ring, &h->ev_near})
        CK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    for (int s = 0; s < GEO_SETS; ++s) {
        CK(cudaEventCreateWithFlags(&h->ev_list[s], cudaEventDisableTiming));
        CK(cudaEventCreateWithFlags(&h->ev_fact[s], cudaEventDisableTiming));
    }
    CK(cudaMallocHost((void**)&h->pinned, sizeof(double) * 4096));
    h->pinned_n = 4096;
    if (c.precision != LBM_PRECISION_FP64) {
        h->fc = h->d.fc = fused_consts(d);
#ifndef LBM_BULK_TILED
#define LBM_BULK_TILED 1
#endif
        h->tmap_ok = LBM_BULK_TILED != 0;
        for (int k = 0; k < 3; ++k) h->tmap_ok = h->tmap_ok && fused_tensor_map(d, h->planes[k], &h->tmap[k]) == 0;
        // two-step passes need the tiled loads and a lattice of a few tiles
        h->pass_ok = c.nx >= 16 && c.ny >= 16 && pass_prepare() == cudaSuccess;
        for (int k = 0; k < 3; ++k)
            h->pass_ok = h->pass_ok && pass_tensor_map(d, h->planes[k], h->d.pass_rows, &h->ptmap[k]) == 0;
    }
    if (init_state(h)) return -1;
    return 0;
}

int lbm_reset(LbmHandle* h) {
    DeviceLock lock(g_device_mutex);
    if (!h) return -1;
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaDeviceSynchronize());
    return init_state(h);
}

int lbm_set_motion_table(LbmHandle* h, const double* rows, int64_t nrows, int32_t ncols) {
    DeviceLock lock(g_device_mutex);
    if (!h) return -1;
    const int nc = 1 + 9 * h->cfg.wing_count;
    if (ncols != nc) return fail(h, "motion table needs 1 + 9*wing_count columns");
    if (nrows < 1 || !rows) return fail(h, "motion table is empty");
    for (int64_t i = 1; i < nrows; ++i)
        if (rows[i * nc] < rows[(i - 1) * nc]) return fail(h, "motion table times must be non-decreasing");
    h->table.assign(rows, rows + (size_t)nrows * nc);
    h->table_rows = nrows;
    h->motion_index = 1;
    // build_motion_step_table (mode.f90:388-412)
    const double dt = h->cfg.scale * h->cfg.uu;
    const double end_time = h->table[(size_t)(nrows - 1) * nc];
    const int64_t steps = (int64_t)((end_time + 1.0e-12) / dt) + 1;
    std::vector<double> st((size_t)steps * nc);
    for (int64_t i = 1; i <= steps; ++i) lookup_motion_row(h, (double)(i - 1) * dt, &st[(size_t)(i - 1) * nc]);
    CK(cudaSetDevice(h->cfg.device));
    if (h->d_step_table) {
        cudaFree(h->d_step_table);
        h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->d_step_table), h->allocs.end());
    }
    if (dalloc(h, &h->d_step_table, st.size())) return -1;
    CK(cudaMemcpy(h->d_step_table, st.data(), st.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaStreamSynchronize(nullptr));   // the copy lands before any step on the handle's streams
    h->d.step_table = h->d_step_table;
    h->geo_ready = -1;
    drop_graphs(h);
    h->d.step_rows = steps;
    h->d.motion_dt = dt;
    return 0;
}

int lbm_set_stream_rows(LbmHandle* h, const double* start_row, const double* target_row) {
    if (!h || !start_row || !target_row) return -1;
    const int nc = h->d.ncol;
    CK(cudaSetDevice(h->cfg.device));
    std::memcpy(h->pinned, start_row, nc * sizeof(double));
    std::memcpy(h->pinned + nc, target_row, nc * sizeof(double));
    CK(cudaMemcpyAsync(h->d.stream_start, h->pinned, nc * sizeof(double), cudaMemcpyHostToDevice, h->s_main));
    CK(cudaMemcpyAsync(h->d.stream_target, h->pinned + nc, nc * sizeof(double), cudaMemcpyHostToDevice, h->s_main));
    CK(cudaStreamSynchronize(h->s_main));
    h->geo_ready = -1;   // the geometry built ahead followed the previous rows
    return 0;
}

int lbm_build_stream_target_row(const LbmHandle* h, const double* start_row, double target_time,
                                const double* delta_row, double* target_row) {
    if (!h) return -1;
    const double dt = target_time - start_row[0];
    if (dt < -1.0e-12) return -2;
    const int nc = 1 + 9 * h->cfg.wing_count;
    std::memcpy(target_row, start_row, nc * sizeof(double));
    target_row[0] = target_time;
    for (int w = 0; w < h->cfg.wing_count; ++w) {
        const int col = 1 + 9 * w, dcol = 1 + 3 * w;
        for (int t = 0; t < 3; ++t) {
            const int cc = col + 3 * t;
            triplet(start_row[cc], start_row[cc + 1], start_row[cc + 1] + delta_row[dcol + t], dt, std::max(dt, 0.0),
                    &target_row[cc], &target_row[cc + 1], &target_row[cc + 2]);
        }
    }
    return 0;
}

int lbm_step(LbmHandle* h, int64_t first_cycle, int64_t n_steps, double* force_rows, int32_t flags) {
    if (!h) return -1;
    if (n_steps < 0) return fail(h, "n_steps must be >= 0");
    if (first_cycle < 1) return fail(h, "cycles start at 1");
    if (h->d.motion_source == LBM_MOTION_FILE && h->d.step_rows <= 0 && h->cfg.wing_count > 0)
        return fail(h, "no motion table loaded");
    CK(cudaSetDevice(h->cfg.device));
    if (ensure_rows(h, n_steps)) return -1;
    const bool fused = h->d.precision != 0;
    // The counters (cycle, the geometry's cycle) are written only when the
    // call does not continue where the last one ended, and then from pinned
    // memory without a host wait (the previous call ended with a stream
    // synchronisation, so the staging words are free).  On the fused path
    // the last step of every call builds the next step's geometry; a
    // continuing call starts from it, any other call builds its first
    // geometry before its first step.
    const bool cont = first_cycle == h->next_cycle;
    const bool have_geo = fused && cont && h->geo_ready == first_cycle;
    long long* stage = reinterpret_cast<long long*>(h->pinned + h->pinned_n - 2);
    if (!cont && n_steps > 0) {
        stage[0] = (long long)first_cycle;
        CK(cudaMemcpyAsync(h->d.cycle, &stage[0], sizeof(long long), cudaMemcpyHostToDevice, h->s_main));
    }
    if (!have_geo && n_steps > 0) {
        stage[1] = (long long)first_cycle;
        CK(cudaMemcpyAsync(h->d.gcycle, &stage[1], sizeof(long long), cudaMemcpyHostToDevice, h->s_main));
    }
    CK(cudaMemsetAsync(h->d.row_index, 0, sizeof(long long), h->s_main));
    if (n_steps > 0) h->next_cycle = h->geo_ready = -1;   // until the steps are enqueued
    const bool want_fields = (flags & LBM_STEP_FIELDS) != 0;
    const bool want_err = (flags & LBM_STEP_ERR) != 0;
    // steps run as two-step passes replayed from CUDA graphs, the last pass
    // launched directly (it computes the residual diagnostic); single steps
    // remain for an odd count and, when the call writes fields or the
    // erranalysis pair, for its last two steps.  Without passes, all but
    // the last two steps replay graphs of GRAPH_STEPS single steps.
    const bool graphs = !h->timing && !(h->cfg.flags & LBM_FLAG_NO_GRAPHS);
    const bool passes = fused && h->pass_ok && !(h->cfg.flags & LBM_FLAG_SINGLE_STEPS);
    if (fused && n_steps > 0 && !have_geo) prime_geometry(h);
    int64_t n = 0;
    if (passes) {
        const int64_t tail = (want_fields || want_err) ? 2 : (n_steps & 1);   // single steps at the end
        // every pass graph a handle can meet (the current planes alternate
        // between two copies, the overlay copy stays, four geometry sets) is
        // built by the first call that replays one, so later calls capture
        // nothing
        if (graphs && n_steps - tail >= 4)
            for (int q = 0; q < 2 * GEO_SETS; ++q) {
                const int c = (q & 1) ? third_planes(h) : h->cur, g = (h->gset + q / 2) % GEO_SETS;
                if (!h->pexec[c][h->alt][g] && build_graph(h, c, h->alt, g, true)) return -1;
            }
        for (; n + 2 <= n_steps - tail; n += 2) {
            const bool last = n + 2 == n_steps;
            if (!graphs || last) {
                enqueue_pass(h, last);
                CK(cudaGetLastError());
                continue;
            }
            wait_pending(h);
            cudaGraphExec_t& ge = h->pexec[h->cur][h->alt][h->gset];
            if (!ge && build_graph(h, h->cur, h->alt, h->gset, true)) return -1;
            CK(cudaGraphLaunch(ge, h->s_main));
            h->cur = third_planes(h);   // as enqueue_pass leaves the state
            h->last_gset = (h->gset + 1) % GEO_SETS;
            h->gset = (h->gset + 2) % GEO_SETS;
        }
    } else if (graphs && fused) {
        // whole graphs while the last two steps stay outside
        for (; n + GRAPH_STEPS <= n_steps - 2; n += GRAPH_STEPS) {
            wait_pending(h);
            cudaGraphExec_t& ge = h->gexec[h->cur][h->alt][h->gset];
            if (!ge && build_graph(h, h->cur, h->alt, h->gset, false)) return -1;
            CK(cudaGraphLaunch(ge, h->s_main));
            h->last_gset = (h->gset + GEO_SETS - 1) % GEO_SETS;
        }
    }
    for (; n < n_steps; ++n) {
        const bool last = n == n_steps - 1, second_last = n == n_steps - 2;
        bool fields = false;
        if (h->d.precision != 0 && ((want_fields && last) || (want_err && (last || second_last)))) {
            // fused path: materialise rho, u, v for this step
            if (!h->d.fo_rho) {
                const size_t N = (size_t)h->d.plane;
                if (dalloc(h, &h->d.fo_rho, N) || dalloc(h, &h->d.fo_u, N) || dalloc(h, &h->d.fo_v, N) ||
                    dalloc(h, &h->d.fo_u0, N) || dalloc(h, &h->d.fo_v0, N))
                    return -1;
            }
            if (want_err && last) {   // previous step's velocity becomes u0
                std::swap(h->d.fo_u, h->d.fo_u0);
                std::swap(h->d.fo_v, h->d.fo_v0);
            }
            fields = true;
        }
        enqueue_step(h, fields, last, true, false);
        CK(cudaGetLastError());
    }
    CK(cudaStreamSynchronize(h->s_main));
    CK(cudaGetLastError());
    if (n_steps > 0) {
        h->next_cycle = first_cycle + n_steps;
        h->geo_ready = fused ? first_cycle + n_steps : -1;
    }
    if (h->timing) collect_phase_times(h);
    if (force_rows && n_steps > 0)
        CK(cudaMemcpy(force_rows, h->d_rowbuf, sizeof(double) * h->row_len * n_steps, cudaMemcpyDeviceToHost));
    if (n_steps > 0) {
        h->fields_valid = h->d.precision == 0 || want_fields || want_err;
        h->err_valid = h->d.precision == 0 ? true : (want_err && n_steps >= 2);
    }
    return check_status(h);
}

int lbm_batch_create(int32_t device, LbmBatch** out) {
    DeviceLock lock(g_device_mutex);
    if (!out) return -1;
    LbmBatch* b = new LbmBatch();
    *out = b;
    b->device = device;
    BCK(cudaSetDevice(device));
    int lo = 0, hi = 0;
    BCK(cudaDeviceGetStreamPriorityRange(&lo, &hi));
    const int mid = (lo + hi) / 2;
    b->prio_lo = lo;
    b->prio_mid = mid;
    b->prio_hi = hi;
    BCK(cudaStreamCreateWithPriority(&b->s_bulk, cudaStreamNonBlocking, lo));
    for (cudaStream_t* st : {&b->s_main, &b->s_ibm})
        BCK(cudaStreamCreateWithPriority(st, cudaStreamNonBlocking, hi));
    for (cudaStream_t* st : {&b->s_bc, &b->s_aux, &b->s_aux2})
        BCK(cudaStreamCreateWithPriority(st, cudaStreamNonBlocking, mid));
    for (cudaEvent_t* e : {&b->ev_start, &b->ev_bulk, &b->ev_ibm, &b->ev_bc, &b->ev_geom, &b->ev_list, &b->ev_fact})
        BCK(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
    for (cudaEvent_t& e : b->ev_tune) BCK(cudaEventCreate(&e));
    return 0;
}

const char* lbm_batch_last_error(const LbmBatch* b) { return b ? b->err.c_str() : "null batch"; }

int lbm_batch_step(LbmBatch* b, int32_t n, LbmHandle* const* hs, const int64_t* first_cycle,
                   const int64_t* n_steps, double* const* force_rows, const int32_t* flags, int32_t* rcs) {
    if (!b) return -1;
    if (n < 0 || (n > 0 && (!hs || !first_cycle || !n_steps))) return batch_fail(b, "bad arguments");
    if (rcs)
        for (int i = 0; i < n; ++i) rcs[i] = 0;
    if (n == 0) return 0;
    for (int i = 0; i < n; ++i) {
        LbmHandle* h = hs[i];
        const std::string who = "episode " + std::to_string(i) + ": ";
        if (!h) return batch_fail(b, who + "null handle");
        if (h->d.precision == 0) return batch_fail(b, who + "batched steps need the FP32 path");
        if (h->cfg.device != b->device) return batch_fail(b, who + "handle on another device");
        if (n_steps[i] < 0) return batch_fail(b, who + "n_steps must be >= 0");
        if (n_steps[i] > (int64_t)1 << 30) return batch_fail(b, who + "n_steps too large");
        if (first_cycle[i] < 1) return batch_fail(b, who + "cycles start at 1");
        if (h->d.motion_source == LBM_MOTION_FILE && h->d.step_rows <= 0 && h->cfg.wing_count > 0)
            return batch_fail(b, who + "no motion table loaded");
        for (int j = 0; j < i; ++j)
            if (hs[j] == h) return batch_fail(b, who + "handle given twice");
    }
    BCK(cudaSetDevice(b->device));
    const int nh = n;
    std::vector<DevState> var((size_t)nh * BV_COUNT);
    for (int i = 0; i < nh; ++i) {
        LbmHandle* h = hs[i];
        const int32_t fl = flags ? flags[i] : 0;
        const bool want_fields = (fl & LBM_STEP_FIELDS) != 0, want_err = (fl & LBM_STEP_ERR) != 0;
        if (ensure_rows(h, n_steps[i])) return batch_fail(b, "episode " + std::to_string(i) + ": " + h->err);
        if ((want_fields || want_err) && n_steps[i] > 0 && !h->d.fo_rho) {
            const size_t N = (size_t)h->d.plane;
            if (dalloc(h, &h->d.fo_rho, N) || dalloc(h, &h->d.fo_u, N) || dalloc(h, &h->d.fo_v, N) ||
                dalloc(h, &h->d.fo_u0, N) || dalloc(h, &h->d.fo_v0, N))
                return batch_fail(b, "episode " + std::to_string(i) + ": " + h->err);
        }
        // the batch's streams start after the handle's own work
        BCK(cudaStreamSynchronize(h->s_main));
        batch_variants(h, want_fields, want_err, &var[(size_t)i * BV_COUNT]);
    }
    // episodes by decreasing step count: the episodes still stepping at any
    // step are a prefix of this order
    std::vector<int> order(nh);
    for (int i = 0; i < nh; ++i) order[i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) { return n_steps[x] > n_steps[y]; });
    const int64_t K = n_steps[order[0]];
    auto active = [&](int64_t k) {   // episodes stepping at step k
        int a = 0;
        while (a < nh && n_steps[order[a]] > k) ++a;
        return a;
    };
    // block offsets of every packed kernel, in episode order
    std::vector<int> boff((size_t)MK_KINDS * (nh + 1), 0);
    size_t factor_smem = 0, solve_smem = 0;
    for (int k = 0; k < MK_KINDS; ++k)
        for (int e = 0; e < nh; ++e) {
            const long long nb = (long long)boff[(size_t)k * (nh + 1) + e] +
                                 multi_blocks((MultiKernel)k, var[(size_t)order[e] * BV_COUNT + BV_PLAIN]);
            if (nb > INT32_MAX) return batch_fail(b, "batch too large for one launch");
            boff[(size_t)k * (nh + 1) + e + 1] = (int)nb;
        }
    for (int e = 0; e < nh; ++e) {
        factor_smem = std::max(factor_smem, hs[order[e]]->factor_smem);
        solve_smem = std::max(solve_smem, (size_t)hs[order[e]]->d.solve_smem);
    }
    // state-pointer tables of every step (variant indices, reused from two
    // steps earlier while the episode set and flags are unchanged)
    struct StepTab { size_t cur, ahead; int a_cur, a_ahead; };
    std::vector<StepTab> steps((size_t)K);
    std::vector<int> pool;                 // variant indices of all tables
    std::vector<int> sig, last_cur[2], last_ahead[2];
    size_t last_cur_at[2] = {0, 0}, last_ahead_at[2] = {0, 0};
    auto intern = [&](const std::vector<int>& v, std::vector<int>* last, size_t* last_at, int ph) {
        if (!v.empty() && last[ph] == v) return last_at[ph];
        const size_t at = pool.size();
        pool.insert(pool.end(), v.begin(), v.end());
        last[ph] = v;
        last_at[ph] = at;
        return at;
    };
    for (int64_t k = 0, a = active(0); k < K; ++k) {
        const int ph = (int)(k & 1);
        const int an = (k + 1 < K) ? active(k + 1) : 0;
        sig.assign((size_t)a, 0);
        for (int e = 0; e < a; ++e) {
            const int i = order[e];
            const int64_t left = n_steps[i] - 1 - k;
            const int v = left == 0 ? BV_LAST : left == 1 ? BV_SECOND_LAST : BV_PLAIN;
            sig[e] = i * BV_COUNT + v + ph;
        }
        steps[k].cur = intern(sig, last_cur, last_cur_at, ph);
        steps[k].a_cur = (int)a;
        sig.assign((size_t)an, 0);
        for (int e = 0; e < an; ++e) sig[e] = order[e] * BV_COUNT + BV_AHEAD + ph;
        steps[k].ahead = an ? intern(sig, last_ahead, last_ahead_at, ph) : 0;
        steps[k].a_ahead = an;
        a = an ? an : active(k + 1);
    }
    // one upload: states, block offsets, first cycles, pointer tables
    auto up16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
    const size_t off_var = 0, off_boff = up16(var.size() * sizeof(DevState));
    const size_t off_cyc = up16(off_boff + boff.size() * sizeof(int));
    const size_t off_ptr = up16(off_cyc + (size_t)nh * sizeof(long long));
    const size_t total = up16(off_ptr + pool.size() * sizeof(DevState*));
    if (total > b->d_cap || total > b->h_cap) {
        DeviceLock lock(g_device_mutex);
        const size_t cap = std::max(total, (size_t)1 << 20) * 2;
        drop_batch_graphs(b);   // they bake addresses in the old tables
        if (b->d_buf) cudaFree(b->d_buf);
        if (b->h_buf) cudaFreeHost(b->h_buf);
        b->d_buf = nullptr;
        b->h_buf = nullptr;
        b->d_cap = b->h_cap = 0;
        BCK(cudaMalloc((void**)&b->d_buf, cap));
        BCK(cudaMallocHost((void**)&b->h_buf, cap));
        b->d_cap = b->h_cap = cap;
    }
    std::memcpy(b->h_buf + off_var, var.data(), var.size() * sizeof(DevState));
    std::memcpy(b->h_buf + off_boff, boff.data(), boff.size() * sizeof(int));
    long long* cyc = reinterpret_cast<long long*>(b->h_buf + off_cyc);
    for (int i = 0; i < nh; ++i) cyc[i] = (long long)first_cycle[i];
    const DevState** ptrs = reinterpret_cast<const DevState**>(b->h_buf + off_ptr);
    const DevState* dvar = reinterpret_cast<const DevState*>(b->d_buf + off_var);
    for (size_t q = 0; q < pool.size(); ++q) ptrs[q] = dvar + pool[q];
    cudaStream_t sm = b->s_main;
    for (int i = 0; i < nh; ++i) hs[i]->next_cycle = hs[i]->geo_ready = -1;   // until the call completes
    BCK(cudaMemcpyAsync(b->d_buf, b->h_buf, total, cudaMemcpyHostToDevice, sm));
    for (int i = 0; i < nh; ++i) {
        for (long long* c : {hs[i]->d.cycle, hs[i]->d.gcycle})
            BCK(cudaMemcpyAsync(c, b->d_buf + off_cyc + (size_t)i * sizeof(long long), sizeof(long long),
                                cudaMemcpyDeviceToDevice, sm));
        BCK(cudaMemsetAsync(hs[i]->d.row_index, 0, sizeof(long long), sm));
    }
    auto launch = [&](MultiKernel k, size_t at, int ne, cudaStream_t st) {
        if (ne <= 0) return;
        const int* bo = reinterpret_cast<const int*>(b->d_buf + off_boff) + (size_t)k * (nh + 1);
        const int nb = boff[(size_t)k * (nh + 1) + ne];
        if (nb <= 0) return;
        MultiArgs m{reinterpret_cast<const DevState* const*>(b->d_buf + off_ptr) + at, bo, ne};
        const size_t smem = (k == MK_FACTOR_SMEM || k == MK_FACTOR_GLOBAL) ? factor_smem : solve_smem;
        if (!launch_multi_ibm(k, m, nb, st) && !launch_multi_solver(k, m, nb, smem, st)) launch_multi_fused(k, m, nb, st);
    };
    auto geometry = [&](size_t at, int ne, cudaStream_t sa, cudaStream_t sb, bool events) {
        launch(MK_GEOMETRY, at, ne, sa);
        if (events) cudaEventRecord(b->ev_geom, sa);
        for (MultiKernel k : {MK_CLAIM, MK_COUNT, MK_SCAN, MK_LIST}) launch(k, at, ne, sa);
        if (events) {
            cudaEventRecord(b->ev_list, sa);
            cudaStreamWaitEvent(sb, b->ev_geom, 0);
        }
        for (MultiKernel k : {MK_ASSEMBLE, MK_FACTOR_SMEM, MK_FACTOR_GLOBAL}) launch(k, at, ne, sb);
        if (events) cudaEventRecord(b->ev_fact, sb);
    };
    // The packed bulk kernel's runs per block: the tuned choice for this
    // batch shape, else steps 1-6 of a call that keeps the same episodes
    // stepping through step 7 time two steps of each candidate (same bits
    // for every choice) and the fastest is kept for the rest of the call
    // and for later calls on the same shape.
    static const int cand[3] = {MK_BULK1, MK_BULK2, MK_BULK4};
    int bulk = MK_BULK2;
    bool tune = false;
    std::vector<long long> shape;
    if (K >= 8 && steps[1].a_cur == steps[7].a_cur) {
        for (int e = 0; e < steps[1].a_cur; ++e)
            shape.push_back((long long)hs[order[e]]->d.nx * 1000003LL + hs[order[e]]->d.ny);
        std::sort(shape.begin(), shape.end());
        const auto it = b->bulk_kind.find(shape);
        if (it != b->bulk_kind.end()) bulk = it->second;
        else tune = true;
    }
    // one packed step, as enqueue_step orders it
    auto emit = [&](const StepTab& t, int kind) {
        cudaEventRecord(b->ev_start, sm);
        for (cudaStream_t st : {b->s_bulk, b->s_ibm, b->s_bc}) cudaStreamWaitEvent(st, b->ev_start, 0);
        if (t.a_ahead) {
            cudaStreamWaitEvent(b->s_aux, b->ev_start, 0);
            geometry(t.ahead, t.a_ahead, b->s_aux, b->s_aux2, true);
        }
        launch(MK_BC, t.cur, t.a_cur, b->s_bc);
        cudaEventRecord(b->ev_bc, b->s_bc);
        for (MultiKernel k2 : {MK_RHS, MK_SOLVE32, MK_SOLVE_SMEM, MK_SOLVE_GLOBAL, MK_SPREAD, MK_FINISH})
            launch(k2, t.cur, t.a_cur, b->s_ibm);
        cudaEventRecord(b->ev_ibm, b->s_ibm);
        launch((MultiKernel)kind, t.cur, t.a_cur, b->s_bulk);
        cudaEventRecord(b->ev_bulk, b->s_bulk);
        cudaStreamWaitEvent(sm, b->ev_bulk, 0);
        cudaStreamWaitEvent(sm, b->ev_ibm, 0);
        cudaStreamWaitEvent(sm, b->ev_bc, 0);
        if (t.a_ahead) {   // the next step's geometry
            cudaStreamWaitEvent(sm, b->ev_list, 0);
            cudaStreamWaitEvent(sm, b->ev_fact, 0);
        }
    };
    // steps from k on in a steady stretch of identical step pairs
    auto same = [&](int64_t x, int64_t y) {
        return steps[x].cur == steps[y].cur && steps[x].ahead == steps[y].ahead && steps[x].a_cur == steps[y].a_cur &&
               steps[x].a_ahead == steps[y].a_ahead;
    };
    std::vector<int64_t> pair_run((size_t)K, 0);
    for (int64_t k = K - 2; k >= 0; --k)
        pair_run[k] = (k + 3 < K && same(k, k + 2) && same(k + 1, k + 3)) ? pair_run[k + 2] + 2 : 2;
    // the geometry of the first step (prime_geometry), then the steps as
    // enqueue_step orders them, every kernel packed over the batch
    if (K > 0) geometry(steps[0].cur, steps[0].a_cur, sm, sm, false);
    for (int64_t k = 0; k < K; ++k) {
        const StepTab& t = steps[k];
        const bool trial = tune && k >= 1 && k <= 6;
        if (trial && (k & 1)) cudaEventRecord(b->ev_tune[(k - 1) / 2], sm);
        if (tune && k == 7) {   // the three trials are done: keep the fastest
            cudaEventRecord(b->ev_tune[3], sm);
            BCK(cudaEventSynchronize(b->ev_tune[3]));
            float best = 0.f;
            for (int c = 0; c < 3; ++c) {
                float ms = 0.f;
                BCK(cudaEventElapsedTime(&ms, b->ev_tune[c], b->ev_tune[c + 1]));
                if (c == 0 || ms < best) {
                    best = ms;
                    bulk = cand[c];
                }
            }
            if (b->bulk_kind.size() > 256) b->bulk_kind.clear();
            b->bulk_kind[shape] = bulk;
            tune = false;
        }
        const int kind = trial ? cand[(k - 1) / 2] : bulk;
        // a steady stretch (the same tables every other step) replays one
        // graph per two steps: captured the first time, kept for later calls
        if (!tune && k + 1 < K) {
            std::vector<long long> key = {(long long)(uintptr_t)b->d_buf, (long long)off_boff, (long long)off_ptr, nh,
                                          (long long)factor_smem, (long long)solve_smem, kind};
            for (int q = 0; q < 2; ++q) {
                const StepTab& u = steps[k + q];
                key.insert(key.end(), {(long long)u.cur, (long long)u.ahead, u.a_cur, u.a_ahead});
            }
            key.insert(key.end(), boff.begin(), boff.end());
            auto it = b->graphs.find(key);
            if (it == b->graphs.end() && pair_run[k] >= GRAPH_PAIR_MIN) {
                if (b->graphs.size() >= 64) drop_batch_graphs(b);
                DeviceLock lock(g_device_mutex);
                cudaGraph_t g = nullptr;
                BCK(cudaStreamBeginCapture(sm, cudaStreamCaptureModeThreadLocal));
                emit(steps[k], kind);
                emit(steps[k + 1], kind);
                BCK(cudaStreamEndCapture(sm, &g));
                cudaGraphExec_t ge = nullptr;
                const cudaError_t e = instantiate_with_priorities(b, g, &ge);
                cudaGraphDestroy(g);
                BCK(e);
                it = b->graphs.emplace(key, ge).first;
            }
            if (it != b->graphs.end()) {
                BCK(cudaGraphLaunch(it->second, sm));
                ++k;   // the pair's second step
                continue;
            }
        }
        emit(t, kind);
    }
    BCK(cudaStreamSynchronize(sm));
    BCK(cudaGetLastError());
    int failed = -1;
    for (int i = 0; i < nh; ++i) {
        LbmHandle* h = hs[i];
        const int64_t ns = n_steps[i];
        const int32_t fl = flags ? flags[i] : 0;
        const bool want_fields = (fl & LBM_STEP_FIELDS) != 0, want_err = (fl & LBM_STEP_ERR) != 0;
        for (bool& q : h->pending) q = false;
        // packed steps leave no geometry built ahead for a later lbm_step
        h->next_cycle = first_cycle[i] + ns;
        h->geo_ready = -1;
        int rc = 0;
        if (ns > 0) {
            if (ns & 1) h->cur = third_planes(h);
            h->last_gset = batch_set(h, (int)((ns - 1) & 1));
            h->gset = batch_set(h, (int)(ns & 1));
            if (want_err) {
                std::swap(h->d.fo_u, h->d.fo_u0);
                std::swap(h->d.fo_v, h->d.fo_v0);
            }
            h->fields_valid = want_fields || want_err;
            h->err_valid = want_err && ns >= 2;
            if (force_rows && force_rows[i]) {
                cudaError_t e = cudaMemcpy(force_rows[i], h->d_rowbuf, sizeof(double) * h->row_len * ns,
                                           cudaMemcpyDeviceToHost);
                if (e != cudaSuccess) rc = cuda_fail(h, e, "cudaMemcpy");
            }
        }
        if (!rc) rc = check_status(h);
        if (rcs) rcs[i] = rc;
        if (rc && failed < 0) failed = i;
    }
    if (failed >= 0) return batch_fail(b, "episode " + std::to_string(failed) + ": " + hs[failed]->err);
    return 0;
}

void lbm_batch_destroy(LbmBatch* b) {
    if (!b) return;
    DeviceLock lock(g_device_mutex);
    cudaSetDevice(b->device);
    for (cudaStream_t s : {b->s_main, b->s_bulk, b->s_ibm, b->s_bc, b->s_aux, b->s_aux2})
        if (s) cudaStreamSynchronize(s);
    drop_batch_graphs(b);
    if (b->d_buf) cudaFree(b->d_buf);
    if (b->h_buf) cudaFreeHost(b->h_buf);
    for (cudaStream_t s : {b->s_main, b->s_bulk, b->s_ibm, b->s_bc, b->s_aux, b->s_aux2})
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : {b->ev_start, b->ev_bulk, b->ev_ibm, b->ev_bc, b->ev_geom, b->ev_list, b->ev_fact})
        if (e) cudaEventDestroy(e);
    for (cudaEvent_t e : b->ev_tune)
        if (e) cudaEventDestroy(e);
    delete b;
}

int lbm_get_sums(LbmHandle* h, double* sum_row, int32_t* sample_count, int32_t* row_len) {
    if (!h) return -1;
    CK(cudaSetDevice(h->cfg.device));
    // on the handle's stream: ordered after its steps (its streams do not
    // synchronise with the legacy default stream)
    if (sum_row)
        CK(cudaMemcpyAsync(sum_row, h->d.sum_row, sizeof(double) * h->row_len, cudaMemcpyDeviceToHost, h->s_main));
    if (sample_count)
        CK(cudaMemcpyAsync(sample_count, h->d.sample_count, sizeof(int), cudaMemcpyDeviceToHost, h->s_main));
    CK(cudaStreamSynchronize(h->s_main));
    if (row_len) *row_len = h->row_len;
    return 0;
}

int lbm_reset_sums(LbmHandle* h) {
    if (!h) return -1;
    CK(cudaSetDevice(h->cfg.device));
    // on the handle's stream, so the next step's force row is added after
    // the clear
    CK(cudaMemsetAsync(h->d.sum_row, 0, sizeof(double) * h->row_len, h->s_main));
    CK(cudaMemsetAsync(h->d.sample_count, 0, sizeof(int), h->s_main));
    return 0;
}

int lbm_get_fields(LbmHandle* h, double* rho, double* u, double* v, double* pre) {
    if (!h) return -1;
    if (!h->fields_valid) return fail(h, "fields are not available: step with LBM_STEP_FIELDS first");
    CK(cudaSetDevice(h->cfg.device));
    const DevState& d = h->d;
    if (d.precision == 0) {
        if (rho && copy_pitched_out(h, d.rho, rho)) return -1;
        if (u && copy_pitched_out(h, d.u, u)) return -1;
        if (v && copy_pitched_out(h, d.v, v)) return -1;
        if (pre && copy_pitched_out(h, d.pre, pre)) return -1;
    } else {
        if (rho && copy_pitched_out(h, d.fo_rho, rho)) return -1;
        if (u && copy_pitched_out(h, d.fo_u, u)) return -1;
        if (v && copy_pitched_out(h, d.fo_v, v)) return -1;
        if (pre) {
            // pre = rho/3 from physical_variables; border nodes keep the
            // value of their never-updated f0 (the BC changes rho, not pre)
            std::vector<double> r((size_t)d.nx * d.ny);
            if (copy_pitched_out(h, d.fo_rho, r.data())) return -1;
            for (size_t k = 0; k < r.size(); ++k) pre[k] = r[k] / 3.0;
            std::vector<double> e(9 * (size_t)(2 * d.nx + 2 * d.ny));
            CK(cudaMemcpy(e.data(), d.edge_f0, e.size() * sizeof(double), cudaMemcpyDeviceToHost));
            const size_t per = 2 * (size_t)d.nx + 2 * (size_t)d.ny;
            auto border_pre = [&](size_t eidx) {
                double s = 0.0;
                for (int k = 0; k < 9; ++k) s = s + e[k * per + eidx];
                return s / 3.0;
            };
            for (int j = 0; j < d.ny; ++j) {
                pre[(size_t)j * d.nx] = border_pre(j);
                pre[(size_t)j * d.nx + d.nx - 1] = border_pre(d.ny + j);
            }
            for (int i = 0; i < d.nx; ++i) {
                pre[i] = border_pre(2 * (size_t)d.ny + i);
                pre[(size_t)(d.ny - 1) * d.nx + i] = border_pre(2 * (size_t)d.ny + d.nx + i);
            }
        }
    }
    return 0;
}

int lbm_get_output(LbmHandle* h, int32_t stride_x, int32_t stride_y, double* u, double* v, double* pre,
                   double* vort) {
    if (!h) return -1;
    if (stride_x < 1 || stride_y < 1) return fail(h, "output strides must be >= 1");
    if (!h->fields_valid) return fail(h, "fields are not available: step with LBM_STEP_FIELDS first");
    CK(cudaSetDevice(h->cfg.device));
    const DevState d = current(h);
    const int onx = (d.nx - 1) / stride_x + 1, ony = (d.ny - 1) / stride_y + 1;
    const size_t per = (size_t)onx * ony;
    if (h->out_cap < 4 * per) {
        DeviceLock lock(g_device_mutex);
        if (h->d_out) {
            cudaFree(h->d_out);
            h->allocs.erase(std::remove(h->allocs.begin(), h->allocs.end(), (void*)h->d_out), h->allocs.end());
            h->dev_bytes -= (int64_t)h->out_cap * sizeof(double);
            h->d_out = nullptr;
            h->out_cap = 0;
        }
        if (dalloc(h, &h->d_out, 4 * per)) return -1;
        h->out_cap = 4 * per;
    }
    launch_output_fields(d, stride_x, stride_y, h->d_out, h->s_main);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->s_main));
    double* dst[4] = {u, v, pre, vort};
    for (int k = 0; k < 4; ++k)
        if (dst[k]) CK(cudaMemcpy(dst[k], h->d_out + k * per, per * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int lbm_err(LbmHandle* h, double* err) {
    if (!h || !err) return -1;
    if (!h->err_valid) return fail(h, "err is not available: step at least twice with LBM_STEP_ERR first");
    CK(cudaSetDevice(h->cfg.device));
    launch_err(current(h), h->err_partial, h->err_out, h->s_main);
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->s_main));
    CK(cudaMemcpy(err, h->err_out, sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

int lbm_get_f(LbmHandle* h, double* f) {
    DeviceLock lock(g_device_mutex);
    if (!h || !f) return -1;
    CK(cudaSetDevice(h->cfg.device));
    const DevState d = current(h);
    const size_t nn = (size_t)d.nx * d.ny;
    if (d.precision == 0) {
        for (int k = 0; k < 9; ++k) {
            CK(cudaMemcpy2D(f + k * nn, sizeof(double) * d.nx, d.f + k * d.plane, sizeof(double) * d.pitch,
                            sizeof(double) * d.nx, d.ny, cudaMemcpyDeviceToHost));
        }
        return 0;
    }
    double* tmp = nullptr;
    CK(cudaMalloc((void**)&tmp, 9 * nn * sizeof(double)));
    launch_fused_export(d, d.gA, tmp, h->s_main);
    cudaError_t e = cudaStreamSynchronize(h->s_main);
    if (e == cudaSuccess) e = cudaMemcpy(f, tmp, 9 * nn * sizeof(double), cudaMemcpyDeviceToHost);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(h, e, "lbm_get_f");
    return 0;
}

int lbm_set_f(LbmHandle* h, const double* f) {
    DeviceLock lock(g_device_mutex);
    if (!h || !f) return -1;
    CK(cudaSetDevice(h->cfg.device));
    const DevState d = current(h);
    const size_t nn = (size_t)d.nx * d.ny;
    if (d.precision == 0) {
        for (int k = 0; k < 9; ++k)
            CK(cudaMemcpy2DAsync(d.f + k * d.plane, sizeof(double) * d.pitch, f + k * nn, sizeof(double) * d.nx,
                                 sizeof(double) * d.nx, d.ny, cudaMemcpyHostToDevice, h->s_main));
        CK(cudaStreamSynchronize(h->s_main));
        return 0;
    }
    double* tmp = nullptr;
    CK(cudaMalloc((void**)&tmp, 9 * nn * sizeof(double)));
    cudaError_t e = cudaMemcpyAsync(tmp, f, 9 * nn * sizeof(double), cudaMemcpyHostToDevice, h->s_main);
    if (e == cudaSuccess) {
        launch_fused_import(d, tmp, d.gA, h->s_main);
        e = cudaStreamSynchronize(h->s_main);
    }
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(h, e, "lbm_set_f");
    return 0;
}

int lbm_get_band(LbmHandle* h, int32_t* n, int32_t* ij_wing, int32_t cap) {
    if (!h || !n) return -1;
    CK(cudaSetDevice(h->cfg.device));
    int nb = 0;
    const DevState g = last_geometry(h);
    CK(cudaMemcpy(&nb, g.band_n, sizeof(int), cudaMemcpyDeviceToHost));
    *n = nb;
    if (!ij_wing) return 0;
    const int m = std::min(nb, cap);
    std::vector<int> ij(2 * (size_t)std::max(m, 1)), w(std::max(m, 1));
    if (m > 0) {
        CK(cudaMemcpy(ij.data(), g.band_ij, 2 * m * sizeof(int), cudaMemcpyDeviceToHost));
        CK(cudaMemcpy(w.data(), g.band_wing, m * sizeof(int), cudaMemcpyDeviceToHost));
    }
    for (int b = 0; b < m; ++b) {
        ij_wing[3 * b] = ij[2 * b] + 1;
        ij_wing[3 * b + 1] = ij[2 * b + 1] + 1;
        ij_wing[3 * b + 2] = w[b] + 1;
    }
    return nb <= cap ? 0 : fail(h, "band larger than cap");
}

int lbm_get_markers(LbmHandle* h, double* xb1, double* yb1, double* xb2, double* yb2) {
    if (!h) return -1;
    CK(cudaSetDevice(h->cfg.device));
    const DevState d = last_geometry(h);
    if (xb1 && d.npts) CK(cudaMemcpy(xb1, d.xb1, d.npts * sizeof(double), cudaMemcpyDeviceToHost));
    if (yb1 && d.npts) CK(cudaMemcpy(yb1, d.yb1, d.npts * sizeof(double), cudaMemcpyDeviceToHost));
    if (xb2 && d.nseg) CK(cudaMemcpy(xb2, d.xb2, d.nseg * sizeof(double), cudaMemcpyDeviceToHost));
    if (yb2 && d.nseg) CK(cudaMemcpy(yb2, d.yb2, d.nseg * sizeof(double), cudaMemcpyDeviceToHost));
    return 0;
}

// Border f0: the fused path keeps it in edge_f0; the plain path in the
// border entries of its f0 planes (interior f0 is rewritten every step).
static int border_f0_copy(LbmHandle* h, double* host, bool to_device) {
    const DevState& d = h->d;
    const long long per = 2LL * d.ny + 2LL * d.nx;
    if (d.precision != 0) {
        const size_t bytes = 9 * (size_t)per * sizeof(double);
        CK(to_device ? cudaMemcpy(d.edge_f0, host, bytes, cudaMemcpyHostToDevice)
                     : cudaMemcpy(host, d.edge_f0, bytes, cudaMemcpyDeviceToHost));
        return 0;
    }
    for (int k = 0; k < 9; ++k) {
        double* plane = d.f0 + k * d.plane;
        double* e = host + k * per;
        const size_t dp = sizeof(double) * d.pitch, one = sizeof(double);
        // columns: one element per row; rows: contiguous
        if (to_device) {
            CK(cudaMemcpy2D(plane, dp, e, one, one, d.ny, cudaMemcpyHostToDevice));
            CK(cudaMemcpy2D(plane + d.nx - 1, dp, e + d.ny, one, one, d.ny, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(plane, e + 2 * d.ny, one * d.nx, cudaMemcpyHostToDevice));
            CK(cudaMemcpy(plane + (long long)(d.ny - 1) * d.pitch, e + 2 * d.ny + d.nx, one * d.nx,
                          cudaMemcpyHostToDevice));
        } else {
            CK(cudaMemcpy2D(e, one, plane, dp, one, d.ny, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy2D(e + d.ny, one, plane + d.nx - 1, dp, one, d.ny, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(e + 2 * d.ny, plane, one * d.nx, cudaMemcpyDeviceToHost));
            CK(cudaMemcpy(e + 2 * d.ny + d.nx, plane + (long long)(d.ny - 1) * d.pitch, one * d.nx,
                          cudaMemcpyDeviceToHost));
        }
    }
    return 0;
}

int lbm_get_border_f0(LbmHandle* h, double* f0, int32_t* movenum) {
    DeviceLock lock(g_device_mutex);
    if (!h) return -1;
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaDeviceSynchronize());
    if (f0 && border_f0_copy(h, f0, false)) return -1;
    if (movenum) *movenum = h->d.movenum;
    return 0;
}

int lbm_set_border_f0(LbmHandle* h, const double* f0, int32_t movenum) {
    DeviceLock lock(g_device_mutex);
    if (!h) return -1;
    CK(cudaSetDevice(h->cfg.device));
    CK(cudaDeviceSynchronize());
    if (f0 && border_f0_copy(h, const_cast<double*>(f0), true)) return -1;
    CK(cudaDeviceSynchronize());   // the copies land before any step on the handle's streams
    h->d.movenum = movenum;
    h->geo_ready = -1;
    drop_graphs(h);   // movenum is baked into the step graphs
    return 0;
}

int lbm_move_mesh(LbmHandle* h, int32_t dr) {
    DeviceLock lock(g_device_mutex);
    if (!h) return -1;
    if (dr != 1 && dr != -1) return fail(h, "dr must be +1 or -1");
    CK(cudaSetDevice(h->cfg.device));
    if (h->d.precision == 0) {
        launch_plain_shift(h->d, dr, h->s_main);
    } else {
        launch_fused_shift(current(h), dr, h->s_main);
        h->cur = third_planes(h);
    }
    CK(cudaGetLastError());
    CK(cudaStreamSynchronize(h->s_main));
    h->d.movenum += dr;
    h->geo_ready = -1;
    drop_graphs(h);
    return 0;
}

int lbm_ibm_residual(LbmHandle* h, double* res) {
    if (!h || !res) return -1;
    CK(cudaSetDevice(h->cfg.device));
    double r[2];
    CK(cudaMemcpy(r, h->d.ibm_resid, sizeof(r), cudaMemcpyDeviceToHost));
    *res = std::sqrt(r[0]) / (std::sqrt(r[1]) + 1e-300);
    return 0;
}

int lbm_status(LbmHandle* h, int32_t* bits) {
    if (!h || !bits) return -1;
    CK(cudaSetDevice(h->cfg.device));
    int st = 0;
    CK(cudaMemcpyAsync(h->pinned + h->pinned_n - 3, h->d.status, sizeof(int), cudaMemcpyDeviceToHost, h->s_main));
    CK(cudaMemsetAsync(h->d.status, 0, sizeof(int), h->s_main));
    CK(cudaStreamSynchronize(h->s_main));
    std::memcpy(&st, h->pinned + h->pinned_n - 3, sizeof(int));
    *bits = st | h->status_seen;
    h->status_seen = 0;
    return 0;
}

int lbm_set_timing(LbmHandle* h, int32_t enable) {
    if (!h) return -1;
    h->timing = enable != 0;
    for (double& v : h->phase_ms) v = 0.0;
    h->timed_steps = 0;
    h->timed_passes = 0;
    if (h->d_far_tiles) {
        CK(cudaSetDevice(h->cfg.device));
        CK(cudaMemsetAsync(h->d_far_tiles, 0, sizeof(int), h->s_main));
        CK(cudaStreamSynchronize(h->s_main));
    }
    h->marks.clear();
    h->evused = 0;
    return 0;
}

int lbm_get_phase_times(LbmHandle* h, double* out, int32_t n) {
    if (!h || !out) return -1;
    double v[10] = {0};
    for (int k = 0; k < 6; ++k) v[k] = h->phase_ms[k];
    v[6] = (double)h->timed_steps;
    v[7] = h->phase_ms[6];
    v[8] = (double)h->timed_passes;
    if (h->d_far_tiles) {
        int ft = 0;
        CK(cudaSetDevice(h->cfg.device));
        CK(cudaMemcpy(&ft, h->d_far_tiles, sizeof(int), cudaMemcpyDeviceToHost));
        v[9] = (double)ft * PASS_TX * h->d.pass_rows;   // nodes of the far tiles
    }
    for (int k = 0; k < n && k < 10; ++k) out[k] = v[k];
    return 0;
}

void* lbm_stream(LbmHandle* h) { return h ? (void*)h->s_main : nullptr; }

int64_t lbm_device_bytes(const LbmHandle* h) { return h ? h->dev_bytes : 0; }

int lbm_mem_info(int32_t device, int64_t* free_bytes, int64_t* total_bytes) {
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return -1;
    if (cudaSetDevice(device) != cudaSuccess) return -1;
    size_t fr = 0, to = 0;
    const cudaError_t e = cudaMemGetInfo(&fr, &to);
    cudaSetDevice(prev);
    if (e != cudaSuccess) return -1;
    if (free_bytes) *free_bytes = (int64_t)fr;
    if (total_bytes) *total_bytes = (int64_t)to;
    return 0;
}

const char* lbm_last_error(const LbmHandle* h) { return h ? h->err.c_str() : "null handle"; }

void lbm_destroy(LbmHandle* h) {
    if (!h) return;
    DeviceLock lock(g_device_mutex);
    cudaSetDevice(h->cfg.device);
    cudaDeviceSynchronize();
    drop_graphs(h);
    for (void* p : h->allocs) cudaFree(p);
    if (h->pinned) cudaFreeHost(h->pinned);
    for (cudaStream_t s :
         {h->s_main, h->s_ibm, h->s_aux[0], h->s_aux[1], h->s_aux2[0], h->s_aux2[1], h->s_bc, h->s_near})
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t e : {h->ev_bc, h->ev_ibm, h->ev_main, h->ev_rhs1, h->ev_chain1, h->ev_bc1, h->ev_ring, h->ev_near})
        if (e) cudaEventDestroy(e);
    for (int s = 0; s < GEO_SETS; ++s) {
        if (h->ev_list[s]) cudaEventDestroy(h->ev_list[s]);
        if (h->ev_fact[s]) cudaEventDestroy(h->ev_fact[s]);
        if (h->ev_geom[s]) cudaEventDestroy(h->ev_geom[s]);
    }
    for (cudaEvent_t e : h->evpool) cudaEventDestroy(e);
    delete h;
}

}  // extern "C"
