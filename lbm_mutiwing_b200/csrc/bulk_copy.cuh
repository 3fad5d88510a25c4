// Bulk copies between global and shared memory through the tensor memory
// accelerator (untiled cp.async.bulk, and tiled tensor loads), completed on
// an mbarrier.
// Addresses must be 16-byte aligned and sizes multiples of 16 bytes.  Every
// wait is bounded: a copy that does not complete within the limit makes the
// caller report an error instead of spinning forever.
#pragma once
#include <cstdint>

namespace lbm {

constexpr long long MBAR_WAIT_LIMIT = 1LL << 22;   // try_wait polls before giving up

__device__ inline uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ inline void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

// One arrival that also announces the bytes the pending copies will deliver.
__device__ inline void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ inline void bulk_load(void* dst_smem, const void* src, uint32_t bytes, uint64_t* bar) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst_smem)),
                 "l"(src), "r"(bytes), "r"(smem_u32(bar))
                 : "memory");
}

// Copies bytes (a multiple of 16) in pieces of at most 64 KB.
__device__ inline void bulk_load_all(void* dst_smem, const void* src, long long bytes, uint64_t* bar) {
    char* d = static_cast<char*>(dst_smem);
    const char* s = static_cast<const char*>(src);
    for (long long o = 0; o < bytes; o += 65536) {
        const long long n = bytes - o < 65536 ? bytes - o : 65536;
        bulk_load(d + o, s + o, (uint32_t)n, bar);
    }
}

// Tiled tensor load of one box of a 3-D tensor map (this GPU's memory; no
// multicast) at coordinates (x, y, z) into shared memory, completed on bar.
// x times the element size must be a multiple of 16 bytes; dst 128-byte
// aligned.
__device__ inline void tma_load_3d(void* dst, const void* tmap, int x, int y, int z, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], "
        "[%5];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
        : "memory");
}

// Waits for the barrier phase with the given parity; false after the limit.
__device__ inline bool mbar_wait(uint64_t* bar, uint32_t parity) {
    for (long long it = 0; it < MBAR_WAIT_LIMIT; ++it) {
        uint32_t ok;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(smem_u32(bar)), "r"(parity)
            : "memory");
        if (ok) return true;
    }
    return false;
}

// Makes this thread's earlier shared-memory writes visible to bulk copies.
__device__ inline void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// Shared -> global bulk store of bytes (a multiple of 16) in 64 KB pieces,
// then waits until the writes are complete.
__device__ inline void bulk_store_all(void* dst, const void* src_smem, long long bytes) {
    char* d = static_cast<char*>(dst);
    const char* s = static_cast<const char*>(src_smem);
    for (long long o = 0; o < bytes; o += 65536) {
        const long long n = bytes - o < 65536 ? bytes - o : 65536;
        asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(d + o),
                     "r"(smem_u32(s + o)), "r"((uint32_t)n)
                     : "memory");
    }
    asm volatile("cp.async.bulk.commit_group;" ::: "memory");
    asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}

}  // namespace lbm
