// Shared device helpers for the FUGAL kernels (sm_100a).
//
// Everything here is generic: warp reductions, 16-byte vector loads of
// fp32 / bf16 / fp16 rows into fp32 registers, mbarrier + bulk-copy wrappers
// (inline PTX) used by the Sinkhorn sweep pipeline, and the bounded-wait
// policy: every spin on an mbarrier gives up after a fixed number of polls,
// records an error code in device memory and lets the kernel return.
#pragma once

#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/fugal_b200.h"

#define FUGAL_DEVICE __device__ __forceinline__

namespace fugal {

// A wait on an mbarrier gives up after kWaitLimitNs of %globaltimer time (or
// kMaxPolls probes, whichever comes first); the kernel then records
// FUGAL_DEVICE_TIMEOUT and returns instead of spinning forever.
constexpr uint64_t kWaitLimitNs = 2000000000ull;  // 2 s
constexpr uint32_t kMaxPolls = 1u << 26;
constexpr uint32_t kSuspendHintNs = 20000u;       // per try_wait

FUGAL_DEVICE uint64_t global_timer_ns() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Device-side error word: the first failing wait writes its code here.
FUGAL_DEVICE void report_error(int* flag, int code) {
    if (flag != nullptr) atomicCAS(flag, 0, code);
}

// SinkhornState.lehmann_momentum (cugal/sinkhorn.py:78-88) over the recorded
// errors, with Python list indexing (negative indices count from the end).
FUGAL_DEVICE double lehmann_omega(const double* errors, int len, int eval_freq, int momentum_start) {
    if (momentum_start < 0 || (long long)len * eval_freq < momentum_start) return 1.0;
    const int index = momentum_start / eval_freq;
    if (len < index - 1) return 1.0;
    int i1 = index - 1, i2 = index - 2;
    if (i1 < 0) i1 += len;
    if (i2 < 0) i2 += len;
    if (i1 < 0 || i2 < 0 || i1 >= len || i2 >= len || i1 >= FUGAL_MAX_RECORDED_ERRORS ||
        i2 >= FUGAL_MAX_RECORDED_ERRORS)
        return 1.0;
    double ratio = errors[i1] / errors[i2];
    if (isnan(ratio)) ratio = 0.99;
    ratio = fmin(ratio, 0.99);
    const double power = 1.0 / eval_freq;
    return 2.0 / (1.0 + sqrt(1.0 - pow(ratio, power)));
}

// ---------------------------------------------------------------- reductions
FUGAL_DEVICE float warp_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
FUGAL_DEVICE float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
FUGAL_DEVICE double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Block-wide double sum (result valid in thread 0). `scratch` holds >= 32 doubles.
FUGAL_DEVICE double block_sum(double v, double* scratch) {
    v = warp_sum(v);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) scratch[warp] = v;
    __syncthreads();
    const int nwarps = (blockDim.x + 31) >> 5;
    v = (threadIdx.x < nwarps) ? scratch[threadIdx.x] : 0.0;
    if (warp == 0) v = warp_sum(v);
    __syncthreads();
    return v;
}

// Fast single-precision exp (CUDA's __expf intrinsic, the MUFU path; relative
// error a few ulp, the same primitive the reference kernels use).
FUGAL_DEVICE float fast_exp(float x) { return __expf(x); }

constexpr float kLog2e = 1.4426950408889634f;
constexpr float kLn2 = 0.6931471805599453f;

// 2^x on the MUFU unit (PTX ex2.approx.ftz.f32).
FUGAL_DEVICE float ex2(float x) {
    float y;
    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}

// ------------------------------------------------------- element conversion
template <typename T> struct Vec;  // one 16-byte chunk of T as fp32

template <> struct Vec<float> {
    static constexpr int N = 4;
    FUGAL_DEVICE static void unpack(const uint4& r, float* out) {
        out[0] = __uint_as_float(r.x); out[1] = __uint_as_float(r.y);
        out[2] = __uint_as_float(r.z); out[3] = __uint_as_float(r.w);
    }
};
template <> struct Vec<__nv_bfloat16> {
    static constexpr int N = 8;
    FUGAL_DEVICE static void unpack(const uint4& r, float* out) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            out[2 * i] = __uint_as_float(w[i] << 16);
            out[2 * i + 1] = __uint_as_float(w[i] & 0xffff0000u);
        }
    }
};
template <> struct Vec<__half> {
    static constexpr int N = 8;
    FUGAL_DEVICE static void unpack(const uint4& r, float* out) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            __half2 h = *reinterpret_cast<const __half2*>(&w[i]);
            float2 f = __half22float2(h);
            out[2 * i] = f.x;
            out[2 * i + 1] = f.y;
        }
    }
};

template <typename T> FUGAL_DEVICE T from_float(float x);
template <> FUGAL_DEVICE float from_float<float>(float x) { return x; }
template <> FUGAL_DEVICE __nv_bfloat16 from_float<__nv_bfloat16>(float x) { return __float2bfloat16_rn(x); }
template <> FUGAL_DEVICE __half from_float<__half>(float x) { return __float2half_rn(x); }

// ------------------------------------------------------------ PTX wrappers
FUGAL_DEVICE uint32_t smem_addr(const void* p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

FUGAL_DEVICE void mbar_init(uint64_t* bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count) : "memory");
}
FUGAL_DEVICE void fence_mbarrier_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
FUGAL_DEVICE void fence_proxy_async_smem() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}
FUGAL_DEVICE void mbar_arrive_expect_tx(uint64_t* bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)), "r"(bytes)
                 : "memory");
}
// Probe of phase `parity`: true once that phase has completed.  The thread may
// be suspended for up to `hint_ns` while the phase is pending.
FUGAL_DEVICE bool mbar_try_wait(uint64_t* bar, uint32_t parity, uint32_t hint_ns = kSuspendHintNs) {
    uint32_t ok;
    asm volatile(
        "{\n .reg .pred p;\n"
        " mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], %2, %3;\n"
        " selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_addr(bar)), "r"(parity), "r"(hint_ns)
        : "memory");
    return ok != 0;
}
// Bounded wait: returns false (and records FUGAL_DEVICE_TIMEOUT) if the phase
// does not complete within limit_ns (0: kWaitLimitNs).
FUGAL_DEVICE bool mbar_wait(uint64_t* bar, uint32_t parity, int* err, uint32_t hint_ns = kSuspendHintNs,
                            uint64_t limit_ns = 0) {
    if (mbar_try_wait(bar, parity, hint_ns)) return true;
    const uint64_t limit = limit_ns != 0 ? limit_ns : kWaitLimitNs;
    const uint64_t t0 = global_timer_ns();
    for (uint32_t i = 0; i < kMaxPolls; ++i) {
        if (mbar_try_wait(bar, parity, hint_ns)) return true;
        if (global_timer_ns() - t0 > limit) break;
    }
    report_error(err, FUGAL_DEVICE_TIMEOUT);
    return false;
}

// 1-D bulk copy global -> this CTA's shared memory, completing on `bar`.
// Both addresses 16-byte aligned, bytes a multiple of 16.
FUGAL_DEVICE void bulk_load(void* smem_dst, const void* gmem_src, uint32_t bytes, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_addr(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}

// ------------------------------------------------------------ cluster / DSMEM
FUGAL_DEVICE uint32_t cluster_ctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}
FUGAL_DEVICE uint32_t cluster_nctarank() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%cluster_nctarank;" : "=r"(r));
    return r;
}
FUGAL_DEVICE uint32_t cluster_id_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%clusterid.x;" : "=r"(r));
    return r;
}
FUGAL_DEVICE uint32_t ncluster_x() {
    uint32_t r;
    asm volatile("mov.u32 %0, %%nclusterid.x;" : "=r"(r));
    return r;
}
FUGAL_DEVICE void cluster_sync() {
    asm volatile("barrier.cluster.arrive.release.aligned;\n"
                 "barrier.cluster.wait.acquire.aligned;" ::: "memory");
}
// Address of the same shared variable in CTA `rank` of this cluster.
FUGAL_DEVICE uint32_t map_to_rank(const void* p, uint32_t rank) {
    uint32_t out;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(smem_addr(p)), "r"(rank));
    return out;
}
FUGAL_DEVICE void st_cluster_f32x2(uint32_t addr, float a, float b) {
    asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(addr), "f"(a), "f"(b) : "memory");
}
// Asynchronous store of two floats into (possibly another CTA's) shared memory
// that completes 8 bytes of transaction count on that CTA's mbarrier.
FUGAL_DEVICE void st_async_f32x2(uint32_t remote_addr, float a, float b, uint32_t remote_bar) {
    asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(
                     remote_addr),
                 "f"(a), "f"(b), "r"(remote_bar)
                 : "memory");
}
// Cluster-wide barrier that tolerates divergent threads (no .aligned).
FUGAL_DEVICE void cluster_sync_any() {
    asm volatile("barrier.cluster.arrive.release;\n"
                 "barrier.cluster.wait.acquire;" ::: "memory");
}
FUGAL_DEVICE void mbar_arrive_cluster(uint32_t remote_bar_addr) {
    asm volatile("mbarrier.arrive.release.cluster.shared::cluster.b64 _, [%0];" ::"r"(remote_bar_addr)
                 : "memory");
}

// ------------------------------------------------------ tensor memory (TMEM)
// Allocation is warp-wide (one warp of the CTA); the address lands in shared
// memory.  Columns: a power of two in [32, 512].
FUGAL_DEVICE void tmem_alloc(uint32_t* smem_dst, uint32_t ncols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(smem_dst)),
                 "r"(ncols)
                 : "memory");
}
FUGAL_DEVICE void tmem_relinquish() {
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
FUGAL_DEVICE void tmem_dealloc(uint32_t taddr, uint32_t ncols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
// Ordering of tensor-memory operations around a thread barrier.
FUGAL_DEVICE void tmem_fence_before_sync() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
FUGAL_DEVICE void tmem_fence_after_sync() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
FUGAL_DEVICE void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }

// Warp-wide 16-column forms of the two accesses below.
FUGAL_DEVICE void tmem_st16(uint32_t taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
        "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
        "r"(__float_as_uint(v[15]))
        : "memory");
}
FUGAL_DEVICE void tmem_ld16(uint32_t taddr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15}, [%16];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Warp-wide: lane i of the warp stores v[0..31] into TMEM lane (lane base + i),
// columns [col, col + 32) of `taddr` (lane base in bits 31..16, column in 15..0;
// the warp's lane base is 32 x (warp index mod 4)).
FUGAL_DEVICE void tmem_st32(uint32_t taddr, const float* v) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31, %32};" ::"r"(taddr),
        "r"(__float_as_uint(v[0])), "r"(__float_as_uint(v[1])), "r"(__float_as_uint(v[2])),
        "r"(__float_as_uint(v[3])), "r"(__float_as_uint(v[4])), "r"(__float_as_uint(v[5])),
        "r"(__float_as_uint(v[6])), "r"(__float_as_uint(v[7])), "r"(__float_as_uint(v[8])),
        "r"(__float_as_uint(v[9])), "r"(__float_as_uint(v[10])), "r"(__float_as_uint(v[11])),
        "r"(__float_as_uint(v[12])), "r"(__float_as_uint(v[13])), "r"(__float_as_uint(v[14])),
        "r"(__float_as_uint(v[15])), "r"(__float_as_uint(v[16])), "r"(__float_as_uint(v[17])),
        "r"(__float_as_uint(v[18])), "r"(__float_as_uint(v[19])), "r"(__float_as_uint(v[20])),
        "r"(__float_as_uint(v[21])), "r"(__float_as_uint(v[22])), "r"(__float_as_uint(v[23])),
        "r"(__float_as_uint(v[24])), "r"(__float_as_uint(v[25])), "r"(__float_as_uint(v[26])),
        "r"(__float_as_uint(v[27])), "r"(__float_as_uint(v[28])), "r"(__float_as_uint(v[29])),
        "r"(__float_as_uint(v[30])), "r"(__float_as_uint(v[31]))
        : "memory");
}
// Warp-wide load of the same layout.  The wait for the load is part of the same
// asm statement, so the registers are valid when it returns.
FUGAL_DEVICE void tmem_ld32(uint32_t taddr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];\n\t"
        "tcgen05.wait::ld.sync.aligned;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr)
        : "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

}  // namespace fugal
