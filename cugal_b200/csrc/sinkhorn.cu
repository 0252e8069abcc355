// Log-domain Sinkhorn for the FUGAL Frank-Wolfe step (cugal/sinkhorn.py:90-120).
//
// Reference semantics, per iteration t (0-based):
//     v <- (1-w) v - w * LSE_i(K_ij + u_i)        column update
//     u <- (1-w) u - w * LSE_j(K_ij + v_j)        row update
//     if t % eval_freq == 0 and t != 0: err = sum_j |sum_i exp(K+u+v)_ij - 1|, stop if err < tol
// The reference reads K four times per iteration (two passes per LSE, a
// transposed copy for the columns) and syncs the host after every launch.
//
// Here one kernel ("sweep") does a whole iteration boundary in ONE read of the
// cost: it computes the row update of iteration t and, while each row is still
// in registers, adds the row-normalised plan P_ij = exp(K_ij + u_i + v_j) into
// per-column sums.  Those sums are (a) exactly the column marginals the
// reference's convergence check measures after iteration t and (b) all the
// column update of iteration t+1 needs: v_j <- v_j - w log(colsum_j).  A small
// "finalize" kernel reduces the per-cluster column sums in FP64, records the
// error, takes the stop / momentum decision on the device and leaves
// log(colsum) for the next sweep, which applies it to v when it loads it (so a
// momentum change at an evaluation point affects v_{t+1} as in the reference).
// Only the first column update of a solve is separate: a max-stabilised merge
// of per-panel column (max, sum) partials, which the gradient writes with the
// cost (column_partials) or a pass over the cost computes (column_pass_kernel).
//
// Two sweep kernels share this structure.
//   sweep_kernel (FP32 sweeps, the absorb sweep, and 16-bit sweeps wider than
//   32768 columns): each cluster of C CTAs owns a contiguous block of rows; CTA
//   k of the cluster owns column slice k.  Row slices stream HBM -> shared
//   memory with 1-D bulk copies (cp.async.bulk + mbarrier, several stages in
//   flight); the per-row (max, sum) partials of the C CTAs are exchanged through
//   distributed shared memory (remote stores + remote mbarrier arrives,
//   double-buffered).  Every thread keeps its 16 or 32 columns' running column
//   sums in registers, so the only global writes are one partial row per cluster.
//   row_sweep_kernel (16-bit sweeps up to 32768 columns): one 512-thread CTA per
//   SM owns whole rows, the row normaliser is a CTA barrier, the column sums
//   live in tensor memory (TMEM); see its own comment below.
//
// Precision: the cost arrives "absorbed" (cost32 = K + U_i + V_j with the
// previous solves' duals U, V folded in), so its entries are ~log P and the
// duals handled here are small increments.  With a BF16/FP16 stream the solve
// reads cost32 for the first fp32_warmup_sweeps sweeps (default none), then an
// "absorb" sweep writes the reduced-precision copy cost16 = cost32 + b_j - m_i,
// m_i the row maximum of cost32 + b_j (rounded once; the row dual a_i + m_i
// carries on in the copy's frame), re-absorbed from cost32 every reabsorb_every
// sweeps, and ends with FP32 polish sweeps on cost32.  LSE, duals and sums are FP32; the
// convergence reduction and the step decisions are FP64.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kMaxStages = 8;
constexpr int kMaxCluster = 16;

struct SolveState {
    int it;          // index of the next sweep
    int done;        // set when the current phase has finished
    int final_it;    // index of the last sweep of the current phase
    int n_err;
    unsigned int ticket;
    int status;      // device-side error code (bounded waits)
    int max_it;      // phase ends after sweep max_it - 1
    int check;       // 1: main phase (convergence checks), 0: polish
    int eval_freq;
    int momentum_start;
    int main_final_it;
    int main_n_err;
    int polish_count;
    int exact_next;  // 1: the next sweep reduces rows with the exact (two-barrier) path
    float max_corr;  // max |log colsum| of the current sweep (as float bits, atomicMax)
    int pad1;
    double threshold;
    double omega;
    double err_accum;
    double last_err;
    double main_last_err;
    double polish_err;
    double errors[FUGAL_MAX_RECORDED_ERRORS];
};

// ------------------------------------------------------------------ device

__device__ double lehmann_momentum(const SolveState* st) {
    return lehmann_omega(st->errors, st->n_err, st->eval_freq, st->momentum_start);
}

// End-of-sweep decision (single thread).
__device__ void decide(SolveState* st, double err) {
    const int t = st->it;
    st->last_err = err;
    bool stop = false;
    if (st->check) {
        if (t % st->eval_freq == 0 && t != 0) {
            if (st->n_err < FUGAL_MAX_RECORDED_ERRORS) st->errors[st->n_err] = err;
            st->n_err += 1;
            if (err < st->threshold)
                stop = true;
            else
                st->omega = lehmann_momentum(st);
        }
    } else {
        st->polish_err = err;
        st->polish_count += 1;
    }
    if (!stop && t + 1 >= st->max_it) stop = true;
    if (st->status != 0) stop = true;  // a bounded wait timed out: end the phase
    if (stop) {
        st->done = 1;
        st->final_it = t;
        if (st->check) {
            st->main_final_it = t;
            st->main_n_err = st->n_err;
            st->main_last_err = err;
        }
    }
    st->it = t + 1;
}

struct SweepArgs {
    const void* L;        // cost (element type T), n x ld
    long long ld;
    int n;
    int n_copy;           // columns copied per row (multiple of 16 bytes)
    int slice_w;          // columns per CTA = threads x columns per thread
    int rows_per_cluster;
    int rows_pad;         // rows_per_cluster rounded up to 32 (shared staging of the row duals)
    unsigned suspend_ns;  // mbarrier try_wait suspend-time hint of the sweep's waits
    int stages;
    const float* b_buf;   // [2][n_pad] column duals of consecutive sweeps
    const float* b_off;   // frame offset added to the previous b (nullable)
    const float* logcs;   // log column sums of the previous sweep
    float* b_buf_w;       // same as b_buf (written slot)
    float* a;             // row duals (read for momentum, written)
    const float* a_off;   // frame offset added to the previous a (nullable)
    float* partials;      // [clusters][n_pad]
    long long n_pad;
    SolveState* st;
    void* out16;          // ABSORB: reduced-precision copy written here
    long long ld16;
    float* a_snap;        // ABSORB: absorbed row duals
    float* b_snap;        // ABSORB: absorbed column duals
};

constexpr int kBarBytes = 128;

// Largest |column correction| (nats) after which the next sweep uses the exact
// (max-stabilised) row reduction instead of the previous row normaliser.
constexpr float kFastPathLimit = 30.0f;

// Sum (or max) of one value per lane, the same in every lane.  The sum is lane
// 0's butterfly result broadcast: every warp that reduces the same inputs then
// holds the bit-identical value, so decisions taken on it are CTA-uniform.
FUGAL_DEVICE float lanes_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return __shfl_sync(0xffffffffu, v, 0);
}
FUGAL_DEVICE float lanes_max(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}

// Shared-memory layout of the sweep kernel (byte offsets from the dynamic base):
//   [0, 128)          mbarriers: full[kMaxStages] (stage loaded), xbar[kXSlots] (exchange done)
//   [128, header)     xch[kXSlots][kMaxCluster][WARPS][R] float2: per-warp row partials of every CTA
//   [header, +4 W)    b_s[slice_w]: this sweep's column duals for the CTA's slice
//   then              a_s[rows_pad], stages[stages][R][slice_w] elements of the streamed cost
constexpr int kXSlots = 2;
template <int THREADS, int R>
__host__ __device__ constexpr int header_bytes_v3() {
    return ((kBarBytes + kXSlots * kMaxCluster * (THREADS / 32) * R * 8) + 127) / 128 * 128;
}

// One cluster-wide all-to-all of per-warp row partials.  Every warp sends its R
// (max, sum) pairs into every CTA of the cluster with st.async (lanes 0..C-1 in
// parallel, one peer each), completing transaction bytes on the receiver's
// exchange barrier; thread 0 arms its own barrier with the bytes it expects.
// `xuse` counts exchanges (identical on every CTA) and selects slot and phase.
// Returns the slot to read, or -1 if the wait timed out.
template <int THREADS, int R>
__device__ __forceinline__ int exchange(float2* xch, uint64_t* xbar, int C, int rank, int& xuse, const float* m,
                                        const float* sm, int* err, unsigned hint_ns) {
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int slot = xuse & 1;
    const uint32_t parity = static_cast<uint32_t>((xuse >> 1) & 1);
    ++xuse;
    if (threadIdx.x == 0) mbar_arrive_expect_tx(&xbar[slot], static_cast<uint32_t>(C * WARPS * R * 8));
    if (lane < C) {
        const uint32_t bar = map_to_rank(&xbar[slot], lane);
#pragma unroll
        for (int r = 0; r < R; ++r)
            st_async_f32x2(map_to_rank(&xch[((slot * kMaxCluster + rank) * WARPS + warp) * R + r], lane), m[r], sm[r],
                           bar);
    }
    return mbar_wait(&xbar[slot], parity, err, hint_ns) ? slot : -1;
}

// Reductions over the C x WARPS partials of one row held in slot `slot`: every
// lane reads a strided subset, then a butterfly; lane 0's result is broadcast so
// every thread of every CTA holds the bit-identical value.
template <int THREADS, int R>
__device__ __forceinline__ float slot_max(const float2* xch, int slot, int C, int r) {
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31;
    float v = -INFINITY;
    for (int i = lane; i < C * WARPS; i += 32) v = fmaxf(v, xch[(slot * kMaxCluster * WARPS + i) * R + r].x);
    return __shfl_sync(0xffffffffu, lanes_max(v), 0);
}
template <int THREADS, int R>
__device__ __forceinline__ float slot_sum(const float2* xch, int slot, int C, int r) {
    constexpr int WARPS = THREADS / 32;
    const int lane = threadIdx.x & 31;
    float v = 0.f;
    for (int i = lane; i < C * WARPS; i += 32) v += xch[(slot * kMaxCluster * WARPS + i) * R + r].y;
    return lanes_sum(v);
}

// One 16-byte chunk of T as float pairs (elements 2q, 2q+1 in .x, .y).
template <typename T> struct Pairs;
template <> struct Pairs<float> {
    FUGAL_DEVICE static void unpack(const uint4& r, float2* o) {
        o[0] = make_float2(__uint_as_float(r.x), __uint_as_float(r.y));
        o[1] = make_float2(__uint_as_float(r.z), __uint_as_float(r.w));
    }
};
template <> struct Pairs<__nv_bfloat16> {
    FUGAL_DEVICE static void unpack(const uint4& r, float2* o) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = make_float2(__uint_as_float(w[i] << 16), __uint_as_float(w[i] & 0xffff0000u));
    }
};
template <> struct Pairs<__half> {
    FUGAL_DEVICE static void unpack(const uint4& r, float2* o) {
        const uint32_t w[4] = {r.x, r.y, r.z, r.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) o[i] = __half22float2(*reinterpret_cast<const __half2*>(&w[i]));
    }
};

FUGAL_DEVICE float2 ex2_pair(float2 x) { return make_float2(ex2(x.x), ex2(x.y)); }

// 2^x for two lanes on the FMA pipe instead of MUFU (Cody-Waite style
// reduction): k = round(x) by the 1.5 * 2^23 rounding constant, f = x - k in
// [-1/2, 1/2], 2^f by a degree-6 polynomial, and k added to the result's
// exponent bits.  The coefficients were fitted for this file by Lawson's
// iteratively reweighted least squares, minimising the relative error on
// [-1/2, 1/2]: 1.9e-9 in exact arithmetic, under 8e-8 (about 1 ulp) with FP32
// Horner steps -- no worse than ex2.approx.  x is clamped to [-127, 127] (so a
// huge x still gives a huge finite value) and x < -126 gives 0, as
// ex2.approx.ftz flushes results below 2^-126; -inf gives 0.
FUGAL_DEVICE float2 ex2_poly_pair(float2 x) {
    const float2 xc = make_float2(fminf(fmaxf(x.x, -127.f), 127.f), fminf(fmaxf(x.y, -127.f), 127.f));
    const float2 rnd = make_float2(12582912.f, 12582912.f);  // 1.5 * 2^23
    const float2 t = __fadd2_rn(xc, rnd);                     // rnd + round(x)
    const float2 k = __fadd2_rn(t, make_float2(-12582912.f, -12582912.f));
    const float2 f = __ffma2_rn(k, make_float2(-1.f, -1.f), xc);  // x - k, exact
    float2 q = make_float2(1.534581242594868e-4f, 1.534581242594868e-4f);
    q = __ffma2_rn(q, f, make_float2(1.3399930903688073e-3f, 1.3399930903688073e-3f));
    q = __ffma2_rn(q, f, make_float2(9.618489071726799e-3f, 9.618489071726799e-3f));
    q = __ffma2_rn(q, f, make_float2(5.550328642129898e-2f, 5.550328642129898e-2f));
    q = __ffma2_rn(q, f, make_float2(2.4022646248340607e-1f, 2.4022646248340607e-1f));
    q = __ffma2_rn(q, f, make_float2(6.931471824645996e-1f, 6.931471824645996e-1f));
    q = __ffma2_rn(q, f, make_float2(1.f, 1.f));
    // the bits of t are those of rnd plus round(x); rnd's low 9 bits are 0, so
    // (bits(t) << 23) is round(x) << 23 modulo 2^32: round(x) added to the exponent
    float2 y;
    y.x = __int_as_float(__float_as_int(q.x) + (__float_as_int(t.x) << 23));
    y.y = __int_as_float(__float_as_int(q.y) + (__float_as_int(t.y) << 23));
    if (x.x < -126.f) y.x = 0.f;
    if (x.y < -126.f) y.y = 0.f;
    return y;
}

// Sweep kernel.  Each thread owns KPT columns of its CTA's slice as KPT/2
// float pairs and processes R rows per batch; the hot loop runs on Blackwell's
// packed FP32x2 FMA/ADD (fma.rn.f32x2) with the exponentials on MUFU ex2, in
// base-2 units (b_s holds the column duals times log2 e).  At most 128
// registers per thread so two 256-thread CTAs share an SM.
template <typename T, int THREADS, int KPT, int R, bool ABSORB, typename TOUT>
__global__ void __launch_bounds__(THREADS, (THREADS >= 512 ? 1 : 512 / THREADS)) sweep_kernel(const SweepArgs p) {
    constexpr int V = Vec<T>::N;  // elements per 16-byte chunk
    constexpr int G = KPT / V;    // chunks per thread per row
    constexpr int VP = V / 2;     // pairs per chunk
    constexpr int H = KPT / 2;    // pairs per thread per row
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ int abort_s;
    uint64_t* full = reinterpret_cast<uint64_t*>(smem);
    uint64_t* xbar = full + kMaxStages;
    float2* xch = reinterpret_cast<float2*>(smem + kBarBytes);
    float* b_s = reinterpret_cast<float*>(smem + header_bytes_v3<THREADS, R>());
    float* a_s = b_s + p.slice_w;  // previous row duals of this cluster's rows
    unsigned char* stage_base = reinterpret_cast<unsigned char*>(a_s + p.rows_pad);

    SolveState* st = p.st;
    if (*reinterpret_cast<volatile int*>(&st->done)) return;  // uniform: written by an earlier kernel

    const int tid = threadIdx.x;
    const int C = static_cast<int>(cluster_nctarank());
    const int rank = static_cast<int>(cluster_ctarank());
    const int cid = static_cast<int>(cluster_id_x());
    const int n = p.n;
    const int col0 = rank * p.slice_w;
    const int ncopy = max(0, min(p.slice_w, p.n_copy - col0));
    const int nvalid = max(0, min(p.slice_w, n - col0));
    const int row_begin = cid * p.rows_per_cluster;
    const int row_end = min(n, row_begin + p.rows_per_cluster);
    const int nbatch = row_end > row_begin ? (row_end - row_begin + R - 1) / R : 0;
    const int t = st->it;
    const float omega = static_cast<float>(st->omega);
    const bool momentum = omega != 1.0f;
    // the absorb sweep always takes the exact path: it writes the copy centred on the row maximum
    const bool exact_only = ABSORB || st->exact_next != 0 || momentum;  // uniform
    const uint32_t row_bytes = static_cast<uint32_t>(ncopy) * sizeof(T);
    const size_t stage_bytes = static_cast<size_t>(R) * p.slice_w * sizeof(T);
    const float* b_prev = p.b_buf + ((t - 1) & 1) * p.n_pad;
    float* b_out = p.b_buf_w + (t & 1) * p.n_pad;
    const float2 log2e2 = make_float2(kLog2e, kLog2e);

    // Column duals of this sweep: b = b_off + b_prev - w log(colsum_prev); kept as b * log2 e.
    for (int j = tid; j < p.slice_w; j += THREADS) {
        float b = 0.f;
        if (j < nvalid) {
            const int jg = col0 + j;
            b = b_prev[jg] - omega * p.logcs[jg];
            if (p.b_off != nullptr) b += p.b_off[jg];
            if (cid == 0) {
                if (ABSORB) {
                    p.b_snap[jg] = b;
                    b_out[jg] = 0.f;
                } else {
                    b_out[jg] = b;
                }
            }
        }
        // columns past n contribute 2^(-inf) = 0 without any masking in the hot loop
        // 16-bit rows (8 columns per 16-byte chunk): split layout, columns 8g..8g+3 at
        // [4g, 4g+4) and 8g+4..8g+7 at [slice_w/2 + 4g, ...), so consecutive threads read
        // consecutive 16 bytes (no bank conflicts); FP32 rows (4 per chunk) are already so
        const int js = (V == 8) ? (((j & 7) < 4 ? 0 : p.slice_w / 2) + (j >> 3) * 4 + (j & 3)) : j;
        b_s[js] = j < nvalid ? b * kLog2e : -INFINITY;
    }
    // Stage columns [ncopy, slice_w) are never written by the bulk copies: zero
    // them once so that they hold finite values (their b_s is -inf).
    if (ncopy < p.slice_w) {
        const int tail = p.slice_w - ncopy;
        for (int s = 0; s < p.stages; ++s)
            for (int r = 0; r < R; ++r) {
                T* row = reinterpret_cast<T*>(stage_base + s * stage_bytes) + static_cast<size_t>(r) * p.slice_w;
                for (int j = tid; j < tail; j += THREADS) row[ncopy + j] = from_float<T>(0.f);
            }
    }
    // Row duals of the previous sweep (the fast path's exponent reference and
    // the momentum term), read once here instead of on every batch's critical path.
    for (int i = tid; i < row_end - row_begin; i += THREADS) {
        float a = p.a[row_begin + i];
        if (p.a_off != nullptr) a += p.a_off[row_begin + i];
        a_s[i] = a;
    }
    if (tid == 0) {
        for (int s = 0; s < p.stages; ++s) mbar_init(&full[s], 1);
        for (int s = 0; s < kXSlots; ++s) mbar_init(&xbar[s], 1);
        fence_mbarrier_init();
        abort_s = 0;
    }
    __syncthreads();
    cluster_sync();  // every peer's barriers exist before the first remote transaction

    auto issue = [&](int bt, int s) {  // batch bt into stage s (bt % stages == s)
        const int r0 = row_begin + bt * R;
        const int rows = min(R, row_end - r0);
        unsigned char* dst = stage_base + s * stage_bytes;
        mbar_arrive_expect_tx(&full[s], rows * row_bytes);
        if (row_bytes > 0) {
            const T* src = static_cast<const T*>(p.L) + static_cast<size_t>(r0) * p.ld + col0;
            for (int r = 0; r < rows; ++r)
                bulk_load(dst + static_cast<size_t>(r) * p.slice_w * sizeof(T), src + static_cast<size_t>(r) * p.ld,
                          row_bytes, &full[s]);
        }
    };
    int issued = 0;
    if (tid == 0) {
        issued = min(p.stages, nbatch);
        for (int bt = 0; bt < issued; ++bt) issue(bt, bt);
    }
    // Stage s of batch bt is no longer read: refill it with batch bt + stages (thread 0).
    auto release = [&](int bt, int s) {
        if (tid == 0 && bt + p.stages < nbatch) {
            fence_proxy_async_smem();
            issue(bt + p.stages, s);
            ++issued;
        }
    };
    // Failure handling: a timed-out wait aborts the whole CTA.  The absorb
    // variant (which has CTA barriers) agrees through __syncthreads_and; the
    // others through a shared flag every thread checks after each wait.
    auto agree = [&](bool ok) -> bool {
        if (ABSORB) return __syncthreads_and(ok) != 0;
        if (!ok) abort_s = 1;
        return ok && *reinterpret_cast<volatile int*>(&abort_s) == 0;
    };
    // b * log2e for the pairs of chunk g of this thread.
    auto load_b2 = [&](int c, float2* b2) {
#pragma unroll
        for (int q = 0; q < VP; q += 2) {
            const float4 b4 = *reinterpret_cast<const float4*>(
                V == 8 ? b_s + (q == 0 ? 0 : p.slice_w / 2) + (c >> 3) * 4 : b_s + c + 2 * q);
            b2[q] = make_float2(b4.x, b4.y);
            b2[q + 1] = make_float2(b4.z, b4.w);
        }
    };

    float2 acc[H];
#pragma unroll
    for (int h = 0; h < H; ++h) acc[h] = make_float2(0.f, 0.f);

    int xuse = 0;
    bool alive = true;
    int bt = 0;
    // stage and barrier parity of batch bt, advanced per batch (no division in the loop)
    int s_next = 0;
    uint32_t ph_next = 0u;
    for (; bt < nbatch; ++bt) {
        const int s = s_next;
        const uint32_t ph = ph_next;
        if (++s_next == p.stages) {
            s_next = 0;
            ph_next ^= 1u;
        }
        if (!agree(mbar_wait(&full[s], ph, &st->status, p.suspend_ns))) {
            alive = false;
            break;
        }
        const int r0 = row_begin + bt * R;
        const int rows = min(R, row_end - r0);
        const T* stage = reinterpret_cast<const T*>(stage_base + s * stage_bytes);

        float2 e[R][H];
        float anew[R], wr[R], a_old[R];
#pragma unroll
        for (int r = 0; r < R; ++r) a_old[r] = (r < rows) ? a_s[bt * R + r] : 0.f;
        bool fast_ok = false;
        float off[R];  // ABSORB: row offset (nats) folded into the reduced-precision copy
#pragma unroll
        for (int r = 0; r < R; ++r) off[r] = 0.f;
        if (!exact_only) {
            // ---- fast path: exponents relative to the previous row normaliser -a_old:
            //      e = 2^(L log2e + b2 + a_old log2e)
            float sm[R], zero[R];
            float2 s2[R], t2[R], ref2[R];  // two partial sums per row (even / odd pairs) for ILP
#pragma unroll
            for (int r = 0; r < R; ++r) {
                ref2[r] = make_float2(a_old[r] * kLog2e, a_old[r] * kLog2e);
                s2[r] = make_float2(0.f, 0.f);
                t2[r] = make_float2(0.f, 0.f);
                zero[r] = 0.f;
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int c = (g * THREADS + tid) * V;
                float2 b2[VP];
                load_b2(c, b2);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r < rows) {
                        float2 v2[VP];
                        Pairs<T>::unpack(*reinterpret_cast<const uint4*>(stage + static_cast<size_t>(r) * p.slice_w + c),
                                         v2);
#pragma unroll
                        for (int q = 0; q < VP; ++q) {
                            const float2 y = ex2_pair(__ffma2_rn(v2[q], log2e2, __fadd2_rn(b2[q], ref2[r])));
                            e[r][g * VP + q] = y;
                            if (q & 1)
                                t2[r] = __fadd2_rn(t2[r], y);
                            else
                                s2[r] = __fadd2_rn(s2[r], y);
                        }
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float2 u2 = __fadd2_rn(s2[r], t2[r]);
                sm[r] = warp_sum(u2.x + u2.y);
            }
            const int slot = exchange<THREADS, R>(xch, xbar, C, rank, xuse, zero, sm, &st->status, p.suspend_ns);
            if (!agree(slot >= 0)) {
                alive = false;
                break;
            }
            float S[R];
            fast_ok = true;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                S[r] = slot_sum<THREADS, R>(xch, slot, C, r);
                if (r < rows && !(S[r] > 1e-30f && S[r] < 1e30f)) fast_ok = false;  // uniform
            }
            if (fast_ok) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    anew[r] = a_old[r] - __log2f(S[r]) * kLn2;  // -(M_ref + ln S)
                    wr[r] = __frcp_rn(S[r]);
                }
                if (!ABSORB) release(bt, s);
            }
        }
        if (!fast_ok) {
            // ---- exact path (base 2): cluster-wide row maximum first, then the exponentials
            float mx[R], zero[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                mx[r] = -INFINITY;
                zero[r] = 0.f;
            }
#pragma unroll
            for (int g = 0; g < G; ++g) {
                const int c = (g * THREADS + tid) * V;
                float2 b2[VP];
                load_b2(c, b2);
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    if (r < rows) {
                        float2 v2[VP];
                        Pairs<T>::unpack(*reinterpret_cast<const uint4*>(stage + static_cast<size_t>(r) * p.slice_w + c),
                                         v2);
#pragma unroll
                        for (int q = 0; q < VP; ++q) {
                            const float2 x = __ffma2_rn(v2[q], log2e2, b2[q]);
                            e[r][g * VP + q] = x;
                            mx[r] = fmaxf(mx[r], fmaxf(x.x, x.y));
                        }
                    } else {
#pragma unroll
                        for (int q = 0; q < VP; ++q) e[r][g * VP + q] = make_float2(-INFINITY, -INFINITY);
                    }
                }
            }
#pragma unroll
            for (int r = 0; r < R; ++r) mx[r] = warp_max(mx[r]);
            int slot = exchange<THREADS, R>(xch, xbar, C, rank, xuse, mx, zero, &st->status, p.suspend_ns);
            if (!agree(slot >= 0)) {
                alive = false;
                break;
            }
            release(bt, s);  // the stage is not read again: x stays in registers
            float M2[R], sm[R];
#pragma unroll
            for (int r = 0; r < R; ++r) {
                M2[r] = slot_max<THREADS, R>(xch, slot, C, r);
                const float base = (M2[r] == -INFINITY) ? 0.f : M2[r];
                const float2 nb = make_float2(-base, -base);
                if (ABSORB && r < rows) {
                    // cost16 = cost32 + b_j - max_j (cost32 + b_j): the row's largest entry is 0,
                    // so the entries that carry its mass get the finest rounding; rounded once
                    off[r] = base * kLn2;
                    TOUT* dst = static_cast<TOUT*>(p.out16) + static_cast<size_t>(r0 + r) * p.ld16 + col0;
#pragma unroll
                    for (int g = 0; g < G; ++g) {
                        const int c = (g * THREADS + tid) * V;
                        if (c < ncopy) {
                            TOUT o[V];
#pragma unroll
                            for (int q = 0; q < VP; ++q) {
                                const float2 x = e[r][g * VP + q];
                                o[2 * q] = from_float<TOUT>(c + 2 * q < nvalid ? (x.x - base) * kLn2 : -INFINITY);
                                o[2 * q + 1] =
                                    from_float<TOUT>(c + 2 * q + 1 < nvalid ? (x.y - base) * kLn2 : -INFINITY);
                            }
                            *reinterpret_cast<uint2*>(dst + c) = *reinterpret_cast<const uint2*>(o);
                        }
                    }
                }
                float2 ss = make_float2(0.f, 0.f);
#pragma unroll
                for (int h = 0; h < H; ++h) {
                    const float2 y = ex2_pair(__fadd2_rn(e[r][h], nb));
                    e[r][h] = y;
                    ss = __fadd2_rn(ss, y);
                }
                sm[r] = warp_sum(ss.x + ss.y);
            }
            slot = exchange<THREADS, R>(xch, xbar, C, rank, xuse, zero, sm, &st->status, p.suspend_ns);
            if (!agree(slot >= 0)) {
                alive = false;
                break;
            }
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const float S = slot_sum<THREADS, R>(xch, slot, C, r);
                const float lse = (M2[r] + log2f(S)) * kLn2;
                anew[r] = momentum ? (1.f - omega) * a_old[r] - omega * lse : -lse;
                // P = e * 2^(M2) * e^(anew)
                wr[r] = (M2[r] == -INFINITY) ? 0.f : ex2(M2[r] + anew[r] * kLog2e);
            }
        }
        if (rank == 0 && tid < rows) {
            float v = anew[0], o = off[0];
#pragma unroll
            for (int r = 1; r < R; ++r)
                if (tid == r) {
                    v = anew[r];
                    o = off[r];
                }
            if (ABSORB) {
                // frame of the copy: a = a_snap + a16 with a_snap = -(row offset)
                p.a_snap[r0 + tid] = -o;
                p.a[r0 + tid] = v + o;
            } else {
                p.a[r0 + tid] = v;
            }
        }
        // Column sums of the row-normalised plan P_ij = e_ij * w_r.
#pragma unroll
        for (int r = 0; r < R; ++r) {
            if (r < rows) {
                const float2 w2 = make_float2(wr[r], wr[r]);
#pragma unroll
                for (int h = 0; h < H; ++h) acc[h] = __ffma2_rn(e[r][h], w2, acc[h]);
            }
        }
    }

    // Per-cluster column sums of the row-normalised plan.
    float* prow = p.partials + static_cast<size_t>(cid) * p.n_pad + col0;
#pragma unroll
    for (int g = 0; g < G; ++g) {
        const int c = (g * THREADS + tid) * V;
        if (c + V <= nvalid) {
#pragma unroll
            for (int q = 0; q < VP; q += 2)
                *reinterpret_cast<float4*>(prow + c + 2 * q) =
                    make_float4(acc[g * VP + q].x, acc[g * VP + q].y, acc[g * VP + q + 1].x, acc[g * VP + q + 1].y);
        } else {
#pragma unroll
            for (int q = 0; q < VP; ++q) {
                if (c + 2 * q < nvalid) prow[c + 2 * q] = acc[g * VP + q].x;
                if (c + 2 * q + 1 < nvalid) prow[c + 2 * q + 1] = acc[g * VP + q].y;
            }
        }
    }

    // An early exit (timed-out wait) may leave bulk copies in flight: wait for
    // them, again bounded, before the shared memory goes away.
    if (!alive && tid == 0) {
        for (int b = bt; b < issued; ++b)
            if (!mbar_wait(&full[b % p.stages], static_cast<uint32_t>((b / p.stages) & 1), &st->status)) break;
    }

    // No CTA leaves while a peer may still send into its shared memory; the
    // non-aligned form tolerates threads that left the batch loop early.
    cluster_sync_any();
}

// ---------------------------------------------------------------------------
// Row-owned 16-bit sweep (n <= 32768): one 512-thread CTA per SM walks a block
// of whole rows, so the row normaliser is a CTA barrier instead of a cluster
// exchange, and each thread keeps the running column sums of its EPT columns
// in tensor memory (TMEM lane 32 (warp % 4) + lane, columns (warp / 4) EPT ..).
// Rows stream through shared memory in segments of up to 16384 elements
// (32 KB) with bulk copies.  The column duals (b log2 e) of the thread's
// columns sit in TMEM next to its column sums (BT = true, columns
// (THREADS / 128) EPT + (warp / 4) EPT ..), so shared memory serves only the
// streamed cost and more stages fit; or, BT = false, in shared memory for the
// whole row.  Same arithmetic as sweep_kernel: fast path against the
// absorbed frame (one barrier per row), exact max-stabilised path (two more
// barriers) for exact sweeps and for rows whose sum leaves (1e-30, 1e30).
// Waits are bounded; a timed-out wait is agreed at the next barrier
// (__syncthreads_and), so every thread leaves the row loop together.
constexpr int kRowSeg = 16384;  // elements per stage segment

struct RowArgs {
    const void* L;
    long long ld;
    int n;
    int n_copy;          // columns copied per row (multiple of 8)
    int rows_per_cta;
    int stages;
    unsigned suspend_ns;
    const float* b_buf;  // [2][n_pad]
    const float* logcs;
    float* b_buf_w;
    float* a;
    float* partials;     // [ctas][n_pad]
    long long n_pad;
    SolveState* st;
    // Failure-detection test hooks (host environment, see make_row_args): the
    // limit of every bounded wait (0: the 2 s default), and a local row of CTA 0
    // whose first copy is armed for 16 bytes more than it delivers (-1: none),
    // so that the waits on it time out.
    unsigned long long wait_limit_ns;
    int fault_row;
};

// Sum of the 16 per-warp row partials, in a fixed pairwise order (every thread
// computes the bit-identical value).
__device__ __forceinline__ float sum16(const float* r) {
    const float4 a = reinterpret_cast<const float4*>(r)[0], b = reinterpret_cast<const float4*>(r)[1];
    const float4 c = reinterpret_cast<const float4*>(r)[2], d = reinterpret_cast<const float4*>(r)[3];
    return (((a.x + a.y) + (a.z + a.w)) + ((b.x + b.y) + (b.z + b.w))) +
           (((c.x + c.y) + (c.z + c.w)) + ((d.x + d.y) + (d.z + d.w)));
}

// POLY: on the fast path, one exponential pair in every POLY (of the 8 pairs of
// two 8-column chunks) is evaluated on the FMA pipe (ex2_poly_pair) instead of
// MUFU; 0: none.
// CL = 2 (rows wider than one CTA covers, up to 65536 columns): a cluster of two
// CTAs owns each block of rows, CTA k taking columns [k COVER, (k + 1) COVER).
// After each CTA barrier the two CTAs swap their row partial (sum, or maximum
// on the exact path) through distributed shared memory: thread 0 stores it
// into the peer's slot with st.async, completing 8 transaction bytes on the
// peer's slot barrier, and every thread waits (bounded) on its own slot
// barrier.  Both CTAs combine the two values in rank order, so they hold the
// bit-identical row normaliser.  Two slots alternate; a peer reuses a slot only
// after it has received the next exchange, which this CTA sends after a barrier
// that follows every read of the slot.  A timed-out exchange is carried to the
// next barrier vote.
template <typename T, int EPT, int THREADS, bool BT, int POLY, int CL>
__global__ void __launch_bounds__(THREADS, 1) row_sweep_kernel(const RowArgs p) {
    constexpr int kRowThreads = THREADS;
    constexpr int kRowWarps = THREADS / 32;
    constexpr int EPS = EPT > kRowSeg / THREADS ? kRowSeg / THREADS : EPT;  // elements per thread per segment
    constexpr int NSEG = EPT / EPS;
    constexpr int G = EPS / 8;                // 16-byte chunks per thread per segment
    constexpr int SEG = kRowThreads * EPS;    // elements per segment
    constexpr int H = EPT / 2;
    constexpr uint32_t TCOLS = (BT ? 2 : 1) * (THREADS / 128) * EPT;
    static_assert(EPT % 16 == 0 && EPS % 8 == 0, "16-column TMEM chunks, 8-element loads");
    static_assert(G % 2 == 0, "column duals load from TMEM 16 at a time");
    static_assert(kRowWarps == 16, "sum16 reduces 16 warp partials");
    static_assert(SEG <= kRowSeg, "segment larger than a stage");
    static_assert(CL == 1 || (CL == 2 && BT), "two-CTA rows keep the column duals in TMEM");
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ uint64_t full[kMaxStages];
    __shared__ uint64_t xbar[2];
    __shared__ __align__(8) float2 xs[2];
    __shared__ __align__(16) float red_s[2][kRowWarps];
    __shared__ __align__(16) float red_m[2][kRowWarps];
    __shared__ __align__(16) float red_grp[2][4][kRowWarps];
    __shared__ uint32_t tmem_slot;

    SolveState* st = p.st;
    if (*reinterpret_cast<volatile int*>(&st->done)) return;  // uniform

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int n = p.n;
    constexpr int COVER = kRowThreads * EPT;  // columns the threads cover (CL COVER >= n)
    const int rank = CL > 1 ? static_cast<int>(cluster_ctarank()) : 0;
    const int grp = static_cast<int>(blockIdx.x) / CL;  // row block (cluster) index
    const int col0 = rank * COVER;                       // first column of this CTA
    float* b_s = reinterpret_cast<float*>(smem);
    unsigned char* stage_base = smem + (BT ? 0 : static_cast<size_t>(COVER) * 4);
    const size_t stage_bytes = static_cast<size_t>(SEG) * sizeof(T);
    const int row_begin = grp * p.rows_per_cta;
    const int row_end = min(n, row_begin + p.rows_per_cta);
    const int nrows = max(0, row_end - row_begin);
    const int units = nrows * NSEG;
    const int t = st->it;
    const float omega = static_cast<float>(st->omega);
    const bool momentum = omega != 1.0f;
    const bool exact_only = st->exact_next != 0 || momentum;  // uniform
    const float* b_prev = p.b_buf + ((t - 1) & 1) * p.n_pad;
    float* b_out = p.b_buf_w + (t & 1) * p.n_pad;
    const float2 log2e2 = make_float2(kLog2e, kLog2e);

    // column duals of this sweep, b = b_prev - w log(colsum_prev), kept as b log2 e;
    // -inf past n, so those columns contribute exactly 0
    if constexpr (!BT) {
        for (int j = tid; j < COVER; j += kRowThreads) {
            float b = -INFINITY;
            if (j < n) {
                const float bj = b_prev[j] - omega * p.logcs[j];
                if (blockIdx.x == 0) b_out[j] = bj;
                b = bj * kLog2e;
            }
            // split layout: columns 8g..8g+3 at [4g, 4g+4), 8g+4..8g+7 at [COVER/2 + 4g, ...), so the
            // 16-byte reads of consecutive threads (8 columns each) are consecutive: no bank conflicts
            b_s[((j & 7) < 4 ? 0 : COVER / 2) + (j >> 3) * 4 + (j & 3)] = b;
        }
    }
    // stage memory starts finite (columns past n_copy are never copied)
    for (size_t k = tid; k < static_cast<size_t>(p.stages) * SEG; k += kRowThreads)
        reinterpret_cast<T*>(stage_base)[k] = from_float<T>(0.f);
    if (tid == 0) {
        for (int s = 0; s < p.stages; ++s) mbar_init(&full[s], 1);
        mbar_init(&xbar[0], 1);
        mbar_init(&xbar[1], 1);
        fence_mbarrier_init();
    }
    if (warp == 0) {
        tmem_alloc(&tmem_slot, TCOLS);
        tmem_relinquish();
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if constexpr (CL > 1) cluster_sync();  // the peer's slot barriers exist before anything is sent
    const uint32_t tcol = tmem_slot + (static_cast<uint32_t>(32 * (warp & 3)) << 16) +
                          static_cast<uint32_t>((warp >> 2) * EPT);
    // this thread's column duals: element e (segment e / EPS, chunk (e % EPS) / 8) is column
    // (e / EPS) SEG + (((e % EPS) / 8) THREADS + tid) 8 + e % 8
    const uint32_t tb = tcol + static_cast<uint32_t>((THREADS / 128) * EPT);
    {
        float z[16];
#pragma unroll
        for (int k = 0; k < 16; ++k) z[k] = 0.f;
#pragma unroll
        for (int k = 0; k < EPT / 16; ++k) tmem_st16(tcol + 16 * k, z);
    }
    if constexpr (BT) {
#pragma unroll
        for (int k = 0; k < EPT / 16; ++k) {
            float bb[16];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int e = 16 * k + 8 * h;
                const int c = (e / EPS) * SEG + (((e % EPS) / 8) * kRowThreads + tid) * 8;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    float b = -INFINITY;
                    const int j = col0 + c + q;
                    if (j < n) {
                        const float bj = b_prev[j] - omega * p.logcs[j];
                        if (grp == 0) b_out[j] = bj;
                        b = bj * kLog2e;
                    }
                    bb[8 * h + q] = b;
                }
            }
            tmem_st16(tb + 16 * k, bb);
        }
    }
    tmem_wait_st();

    // Stage ring cursor: the stage and barrier parity of the first unit of a row,
    // advanced row by row (no division by the runtime stage count in the loop).
    struct Cursor {
        int s;
        uint32_t ph;
    };
    const int NST = p.stages;
    auto unit_at = [&](Cursor c, int sg, int& st_idx, uint32_t& par_bit) {
        st_idx = c.s + sg;
        par_bit = c.ph;
        if (st_idx >= NST) {
            st_idx -= NST;
            par_bit ^= 1u;
        }
    };
    auto next_rows = [&](Cursor c, int k) {
        c.s += k * NSEG;
        while (c.s >= NST) {
            c.s -= NST;
            c.ph ^= 1u;
        }
        return c;
    };
    Cursor cur{0, 0u};

    auto issue = [&](int u, int s) {  // unit u into stage s (u % S == s)
        const int row = row_begin + u / NSEG;
        const int seg = u % NSEG;
        const int cols = min(SEG, p.n_copy - col0 - seg * SEG);
        const uint32_t bytes = cols > 0 ? static_cast<uint32_t>(cols) * sizeof(T) : 0u;
        const uint32_t unmet = (blockIdx.x == 0 && u == p.fault_row * NSEG) ? 16u : 0u;
        mbar_arrive_expect_tx(&full[s], bytes + unmet);
        if (bytes > 0)
            bulk_load(stage_base + s * stage_bytes,
                      static_cast<const T*>(p.L) +
                          static_cast<unsigned long long>(static_cast<unsigned>(row)) * static_cast<unsigned>(p.ld) +
                          col0 + static_cast<size_t>(seg) * SEG,
                      bytes, &full[s]);
    };
    int issued = 0;
    if (tid == 0) {
        fence_proxy_async_smem();  // the zero fill above precedes the copies
        issued = min(p.stages, units);
        for (int u = 0; u < issued; ++u) issue(u, u);
    }
    auto release = [&](int r, Cursor c) {  // c: the cursor of row r
        if (tid == 0) {
            fence_proxy_async_smem();
            for (int sg = 0; sg < NSEG; ++sg) {
                const int u = r * NSEG + sg + NST;
                if (u < units) {
                    int si;
                    uint32_t ph;
                    unit_at(c, sg, si, ph);
                    issue(u, si);
                    ++issued;
                }
            }
        }
    };
    // Swap of one row partial with the peer CTA (CL = 2); returns the peer's value.
    int xuse = 0;
    bool xok = true;  // every exchange so far completed (voted on at the next barrier)
    auto swap_with_peer = [&](float v) -> float {
        const int slot = xuse & 1;
        const uint32_t parity = static_cast<uint32_t>((xuse >> 1) & 1);
        ++xuse;
        if (tid == 0) {
            mbar_arrive_expect_tx(&xbar[slot], 8u);
            const uint32_t peer = static_cast<uint32_t>(rank ^ 1);
            st_async_f32x2(map_to_rank(&xs[slot], peer), v, 0.f, map_to_rank(&xbar[slot], peer));
        }
        xok = mbar_wait(&xbar[slot], parity, &st->status, p.suspend_ns, p.wait_limit_ns) && xok;
        return xs[slot].x;
    };
    auto b2_at = [&](int c, float2* b2) {  // c: a multiple of 8
        const float4 lo = *reinterpret_cast<const float4*>(b_s + (c >> 3) * 4);
        const float4 hi = *reinterpret_cast<const float4*>(b_s + COVER / 2 + (c >> 3) * 4);
        b2[0] = make_float2(lo.x, lo.y);
        b2[1] = make_float2(lo.z, lo.w);
        b2[2] = make_float2(hi.x, hi.y);
        b2[3] = make_float2(hi.z, hi.w);
    };
    // Column duals of chunks g0 and g0 + 1 of segment sg (16 elements): from TMEM
    // (BT), else from shared memory.  b2[8 * gg + q] holds columns 2q, 2q + 1 of chunk g0 + gg.
    auto b_pair = [&](int sg, int g0, float2 (&b2)[8]) {
        if constexpr (BT) {
            float bb[16];
            tmem_ld16(tb + sg * EPS + g0 * 8, bb);
#pragma unroll
            for (int q = 0; q < 8; ++q) b2[q] = make_float2(bb[2 * q], bb[2 * q + 1]);
        } else {
            b2_at(sg * SEG + (g0 * kRowThreads + tid) * 8, b2);
            b2_at(sg * SEG + ((g0 + 1) * kRowThreads + tid) * 8, b2 + 4);
        }
    };

    // Fast-path exponentials of local row rr (its stages waited for here):
    // yy = 2^(L log2e + b) against the absorbed frame, s2 / t2 partial row sums.
    auto row_fast = [&](Cursor c, float2(&yy)[H], float2& s2, float2& t2, bool& okk) {
#pragma unroll
        for (int sg = 0; sg < NSEG; ++sg) {
            int si;
            uint32_t ph;
            unit_at(c, sg, si, ph);
            okk = mbar_wait(&full[si], ph, &st->status, p.suspend_ns, p.wait_limit_ns) && okk;
            const T* stage = reinterpret_cast<const T*>(stage_base + si * stage_bytes);
#pragma unroll
            for (int g0 = 0; g0 < G; g0 += 2) {
                float2 b2[8];
                b_pair(sg, g0, b2);
#pragma unroll
                for (int gg = 0; gg < 2; ++gg) {
                    const int g = g0 + gg;
                    const int cl = (g * kRowThreads + tid) * 8;
                    float2 v2[4];
                    Pairs<T>::unpack(*reinterpret_cast<const uint4*>(stage + cl), v2);
#pragma unroll
                    for (int q = 0; q < 4; ++q) {
                        const float2 xq = __ffma2_rn(v2[q], log2e2, b2[4 * gg + q]);
                        const float2 e = (POLY > 0 && (4 * gg + q) % (POLY > 0 ? POLY : 1) == (POLY > 0 ? POLY : 1) - 1)
                                             ? ex2_poly_pair(xq)
                                             : ex2_pair(xq);
                        yy[(sg * EPS + g * 8) / 2 + q] = e;
                        if (q & 1)
                            t2 = __fadd2_rn(t2, e);
                        else
                            s2 = __fadd2_rn(s2, e);
                    }
                }
            }
        }
    };

    bool alive = true;
    int r = 0;
    // Rows in groups of RB = 64 / EPT (one-segment rows, fast path): the group's
    // exponentials stay in registers, so its rows share one barrier, one read of
    // the per-warp sums and one pass over the TMEM accumulators.  A group with a
    // row outside the fast path's range hands the rest of the sweep to the
    // single-row loop below, which restarts at that group (stages still held).
    if constexpr (CL == 1 && NSEG == 1 && EPT <= 32) {
        constexpr int RB = 64 / EPT;  // 2 or 4
        if (!exact_only) {
            for (; r < nrows; r += RB) {
                const int nr = min(RB, nrows - r);
                const int par = (r / RB) & 1;
                bool ok = true;
                float2 yg[RB][H];
                float part[RB];
#pragma unroll
                for (int k = 0; k < RB; ++k) {
                    float2 sa = make_float2(0.f, 0.f), ta = sa;
                    if (k < nr) {
                        row_fast(next_rows(cur, k), yg[k], sa, ta, ok);
                    } else {
#pragma unroll
                        for (int h = 0; h < H; ++h) yg[k][h] = make_float2(0.f, 0.f);
                    }
                    const float2 ua = __fadd2_rn(sa, ta);
                    part[k] = ua.x + ua.y;
                }
#pragma unroll
                for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
                    for (int k = 0; k < RB; ++k) part[k] += __shfl_xor_sync(0xffffffffu, part[k], o);
                }
                if (lane == 0) {
#pragma unroll
                    for (int k = 0; k < RB; ++k) red_grp[par][k][warp] = part[k];
                }
                if (!__syncthreads_and(ok)) {
                    alive = false;
                    break;
                }
                float S[RB], wk[RB];
                bool in_range = true;
#pragma unroll
                for (int k = 0; k < RB; ++k) {
                    S[k] = sum16(red_grp[par][k]);
                    if (k < nr && !(S[k] > 1e-30f && S[k] < 1e30f)) in_range = false;
                }
                if (!in_range) break;  // uniform
#pragma unroll
                for (int k = 0; k < RB; ++k) {
                    if (k < nr) release(r + k, next_rows(cur, k));
                    wk[k] = k < nr ? __frcp_rn(S[k]) : 0.f;
                    if (tid == 0 && k < nr) p.a[row_begin + r + k] = -__log2f(S[k]) * kLn2;
                }
#pragma unroll
                for (int c = 0; c < EPT / 16; ++c) {
                    float acc[16];
                    tmem_ld16(tcol + 16 * c, acc);
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        float2 a2 = make_float2(acc[2 * q], acc[2 * q + 1]);
#pragma unroll
                        for (int k = 0; k < RB; ++k) a2 = __ffma2_rn(yg[k][8 * c + q], make_float2(wk[k], wk[k]), a2);
                        acc[2 * q] = a2.x;
                        acc[2 * q + 1] = a2.y;
                    }
                    tmem_st16(tcol + 16 * c, acc);
                }
                cur = next_rows(cur, nr);
            }
        }
    }
    if (alive)
    for (; r < nrows; ++r) {
        const int row = row_begin + r;
        const int par = r & 1;
        const Cursor rc = cur;
        bool ok = true;
        float2 y[H];
        float anew = 0.f, wr = 0.f;
        bool fast_ok = false;
        if (!exact_only) {
            // ---- fast path: 2^(L log2e + b) against the absorbed frame
            float2 s2 = make_float2(0.f, 0.f), t2 = make_float2(0.f, 0.f);
            row_fast(rc, y, s2, t2, ok);
            const float2 u2 = __fadd2_rn(s2, t2);
            const float part = warp_sum(u2.x + u2.y);
            if (lane == 0) red_s[par][warp] = part;
            if (!__syncthreads_and(ok && xok)) {
                alive = false;
                break;
            }
            float S = sum16(red_s[par]);
            if constexpr (CL > 1) {
                const float Sp = swap_with_peer(S);
                S = rank == 0 ? S + Sp : Sp + S;
            }
            fast_ok = S > 1e-30f && S < 1e30f;  // uniform
            if (fast_ok) {
                release(r, rc);
                anew = -__log2f(S) * kLn2;
                wr = __frcp_rn(S);
            }
        }
        if (!fast_ok) {
            // ---- exact path: row maximum, then the exponentials relative to it
            // (the previous row dual is read before any exchange of this row, so a
            // peer that writes it later cannot have written it yet)
            const float a_old = momentum ? p.a[row] : 0.f;
            float mx = -INFINITY;
#pragma unroll
            for (int sg = 0; sg < NSEG; ++sg) {
                int si;
                uint32_t ph;
                unit_at(rc, sg, si, ph);
                if (exact_only) ok = mbar_wait(&full[si], ph, &st->status, p.suspend_ns, p.wait_limit_ns) && ok;
                const T* stage = reinterpret_cast<const T*>(stage_base + si * stage_bytes);
#pragma unroll
                for (int g0 = 0; g0 < G; g0 += 2) {
                    float2 b2[8];
                    b_pair(sg, g0, b2);
#pragma unroll
                    for (int gg = 0; gg < 2; ++gg) {
                        const int g = g0 + gg;
                        const int cl = (g * kRowThreads + tid) * 8;
                        float2 v2[4];
                        Pairs<T>::unpack(*reinterpret_cast<const uint4*>(stage + cl), v2);
#pragma unroll
                        for (int q = 0; q < 4; ++q) {
                            const float2 x = __ffma2_rn(v2[q], log2e2, b2[4 * gg + q]);
                            y[(sg * EPS + g * 8) / 2 + q] = x;
                            mx = fmaxf(mx, fmaxf(x.x, x.y));
                        }
                    }
                }
            }
            mx = warp_max(mx);
            if (lane == 0) red_m[par][warp] = mx;
            if (!__syncthreads_and(ok && xok)) {
                alive = false;
                break;
            }
            float M2 = -INFINITY;
#pragma unroll
            for (int w = 0; w < kRowWarps; ++w) M2 = fmaxf(M2, red_m[par][w]);
            if constexpr (CL > 1) M2 = fmaxf(M2, swap_with_peer(M2));
            const float base = (M2 == -INFINITY) ? 0.f : M2;
            const float2 nb = make_float2(-base, -base);
            float2 ss = make_float2(0.f, 0.f);
#pragma unroll
            for (int h = 0; h < H; ++h) {
                y[h] = ex2_pair(__fadd2_rn(y[h], nb));
                ss = __fadd2_rn(ss, y[h]);
            }
            const float part = warp_sum(ss.x + ss.y);
            if (lane == 0) red_s[par][warp] = part;
            if (!__syncthreads_and(xok)) {
                alive = false;
                break;
            }
            release(r, rc);
            float S = sum16(red_s[par]);
            if constexpr (CL > 1) {
                const float Sp = swap_with_peer(S);
                S = rank == 0 ? S + Sp : Sp + S;
            }
            const float lse = (M2 + log2f(S)) * kLn2;
            anew = momentum ? (1.f - omega) * a_old - omega * lse : -lse;
            wr = (M2 == -INFINITY) ? 0.f : ex2(M2 + anew * kLog2e);
        }
        if (tid == 0 && rank == 0) p.a[row] = anew;
        // column sums of the row-normalised plan, accumulated in TMEM (one 16-column
        // chunk per load; batching two chunks per wait measured slower)
        const float2 w2 = make_float2(wr, wr);
#pragma unroll
        for (int k = 0; k < EPT / 16; ++k) {
            float acc[16];
            tmem_ld16(tcol + 16 * k, acc);
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float2 a2 = __ffma2_rn(y[8 * k + q], w2, make_float2(acc[2 * q], acc[2 * q + 1]));
                acc[2 * q] = a2.x;
                acc[2 * q + 1] = a2.y;
            }
            tmem_st16(tcol + 16 * k, acc);
        }
        cur = next_rows(cur, 1);
    }

    // per-CTA column sums -> partials[cta][col]
    tmem_wait_st();
    float* prow = p.partials + static_cast<size_t>(grp) * p.n_pad + col0;
    const int nloc = n - col0;
#pragma unroll
    for (int k = 0; k < EPT / 16; ++k) {
        float acc[16];
        tmem_ld16(tcol + 16 * k, acc);
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            const int e = 16 * k + 8 * half;  // element index: segment e / EPS, chunk (e % EPS) / 8
            const int c = (e / EPS) * SEG + (((e % EPS) / 8) * kRowThreads + tid) * 8;
            const float* src = acc + 8 * half;
            if (c + 8 <= nloc) {
                *reinterpret_cast<float4*>(prow + c) = make_float4(src[0], src[1], src[2], src[3]);
                *reinterpret_cast<float4*>(prow + c + 4) = make_float4(src[4], src[5], src[6], src[7]);
            } else {
                for (int q = 0; q < 8; ++q)
                    if (c + q < nloc) prow[c + q] = src[q];
            }
        }
    }
    // a timed-out wait may leave copies in flight: wait for each (bounded) before
    // the shared memory they land in is released; the copies of different units
    // complete on different stage barriers, so one that never completes does not
    // hide the others
    if (!alive && tid == 0) {
        for (int u = r * NSEG; u < issued; ++u)
            mbar_wait(&full[u % p.stages], static_cast<uint32_t>((u / p.stages) & 1), &st->status, kSuspendHintNs,
                      p.wait_limit_ns);
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    if (warp == 0) tmem_dealloc(tmem_slot, TCOLS);
    // no CTA leaves while its peer may still send into its shared memory; the
    // non-aligned form tolerates threads that left the row loop early
    if constexpr (CL > 1) cluster_sync_any();
}

// Reduce the per-cluster column sums (FP64), write log(colsum), decide.
// Block: 8 warps x 32 lanes; lanes own 4 consecutive columns each (128 per
// block), warps split the partial rows; one FP64 error sum and one maximum
// |column correction| per block go to the solve state by atomics.
constexpr int kFinThreads = 256;
constexpr int kFinCols = 128;

__global__ void __launch_bounds__(kFinThreads) finalize_kernel(const float* partials, int nparts, long long n_pad,
                                                               int n, float* logcs, SolveState* st) {
    __shared__ double part[kFinThreads / 32][kFinCols];
    __shared__ double red[32];
    __shared__ float red_corr[kFinThreads / 32];
    if (*reinterpret_cast<volatile int*>(&st->done)) return;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int j0 = blockIdx.x * kFinCols + lane * 4;
    double cs[4] = {0.0, 0.0, 0.0, 0.0};
    if (j0 < n) {
        for (int c = warp; c < nparts; c += kFinThreads / 32) {
            const float4 v = *reinterpret_cast<const float4*>(partials + static_cast<size_t>(c) * n_pad + j0);
            cs[0] += v.x; cs[1] += v.y; cs[2] += v.z; cs[3] += v.w;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) part[warp][lane * 4 + q] = cs[q];
    __syncthreads();
    double err = 0.0;
    float corr = 0.f;
    if (threadIdx.x < kFinCols) {
        const int j = blockIdx.x * kFinCols + threadIdx.x;
        if (j < n) {
            double tot = 0.0;
#pragma unroll
            for (int w = 0; w < kFinThreads / 32; ++w) tot += part[w][threadIdx.x];
            err = fabs(tot - 1.0);
            const float lg = static_cast<float>(log(fmax(tot, 1e-37)));
            logcs[j] = lg;
            corr = fabsf(lg);
        }
    }
    corr = warp_max(corr);
    if (lane == 0) red_corr[warp] = corr;
    err = block_sum(err, red);  // contains __syncthreads: red_corr is complete
    if (threadIdx.x == 0) {
        float bc = 0.f;
        for (int w = 0; w < kFinThreads / 32; ++w) bc = fmaxf(bc, red_corr[w]);
        if (bc > 0.f) atomicMax(reinterpret_cast<unsigned int*>(&st->max_corr), __float_as_uint(bc));
        atomicAdd(&st->err_accum, err);
        __threadfence();
        const unsigned prev = atomicAdd(&st->ticket, 1u);
        if (prev == gridDim.x - 1) {
            __threadfence();
            const double total = atomicAdd(&st->err_accum, 0.0);
            const float max_corr = __uint_as_float(atomicOr(reinterpret_cast<unsigned int*>(&st->max_corr), 0u));
            st->err_accum = 0.0;
            st->ticket = 0;
            st->max_corr = 0.f;
            decide(st, total);
            // the next sweep may use the previous row normaliser as its reference
            // only if no column moves by more than kFastPathLimit nats
            st->exact_next = (max_corr * static_cast<float>(st->omega) > kFastPathLimit || st->omega != 1.0) ? 1 : 0;
        }
    }
}

// First column update of a solve, max-stabilised: per (row chunk, column) an
// online (max, sum) of exp(cost_ij + a_i).
__global__ void __launch_bounds__(256) column_pass_kernel(const float* L, long long ld, int n, const float* a,
                                                          int rows_per_chunk, float2* part, long long n_pad) {
    // Per column and row chunk: online (max, sum) of 2^((L_ij + a_i) log2 e), base-2 units,
    // eight rows per step (their loads are all in flight before the exponentials).
    const int j0 = (blockIdx.x * blockDim.x + threadIdx.x) * 4;
    const int chunk = blockIdx.y;
    const int i0 = chunk * rows_per_chunk;
    const int i1 = min(n, i0 + rows_per_chunk);
    if (j0 >= n) return;
    const bool full4 = (j0 + 4 <= n) && ((ld & 3) == 0);
    constexpr int RR = 8;
    float m[4], s[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        m[q] = -INFINITY;
        s[q] = 0.f;
    }
    for (int i = i0; i < i1; i += RR) {
        float x[RR][4];
#pragma unroll
        for (int r = 0; r < RR; ++r) {
            const int row = i + r;
            if (row < i1) {
                const float ai = a[row];
                const float* src = L + static_cast<size_t>(row) * ld + j0;
                if (full4) {
                    const float4 v = *reinterpret_cast<const float4*>(src);
                    x[r][0] = (v.x + ai) * kLog2e; x[r][1] = (v.y + ai) * kLog2e;
                    x[r][2] = (v.z + ai) * kLog2e; x[r][3] = (v.w + ai) * kLog2e;
                } else {
#pragma unroll
                    for (int q = 0; q < 4; ++q) x[r][q] = (j0 + q < n) ? (src[q] + ai) * kLog2e : -INFINITY;
                }
            } else {
#pragma unroll
                for (int q = 0; q < 4; ++q) x[r][q] = -INFINITY;
            }
        }
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float mn = m[q];
#pragma unroll
            for (int r = 0; r < RR; ++r) mn = fmaxf(mn, x[r][q]);
            if (mn == -INFINITY) continue;
            float acc = (m[q] == -INFINITY) ? 0.f : s[q] * ex2(m[q] - mn);
#pragma unroll
            for (int r = 0; r < RR; ++r) acc += ex2(x[r][q] - mn);
            m[q] = mn;
            s[q] = acc;
        }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
        if (j0 + q < n) part[static_cast<size_t>(chunk) * n_pad + j0 + q] = make_float2(m[q], s[q]);
}

struct InitArgs {
    int max_it;
    int eval_freq;
    int momentum_start;
    double threshold;
};

// Merge base-2 column partials (max, sum) into v_0 = -LSE_i(cost + a) (momentum
// is 1 at iteration 0), stored as the "previous sweep" b, with a zero pending
// correction; block 0 also resets the solve state.  A block takes 32 columns;
// its 8 warps split the chunks (each a two-pass max-then-sum), then warp 0
// combines the 8 pairs.  Grid: ceil(n / 32) blocks of 256 threads.
constexpr int kMergeLanes = 8;
__global__ void __launch_bounds__(256) column_merge_kernel(const float2* part, int nchunks, long long part_ld,
                                                           long long n_pad, int n, float* b_buf, float* logcs,
                                                           SolveState* st, InitArgs ia) {
    __shared__ float2 red[kMergeLanes][32];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->it = 0;
        st->done = 0;
        st->final_it = -1;
        st->n_err = 0;
        st->ticket = 0;
        st->status = 0;
        st->max_it = ia.max_it;
        st->check = 1;
        st->eval_freq = ia.eval_freq;
        st->momentum_start = ia.momentum_start;
        st->main_final_it = -1;
        st->main_n_err = 0;
        st->polish_count = 0;
        st->exact_next = 1;
        st->max_corr = 0.f;
        st->threshold = ia.threshold;
        st->omega = 1.0;
        st->err_accum = 0.0;
        st->last_err = 0.0;
        st->main_last_err = 0.0;
        st->polish_err = 0.0;
    }
    const int lane = threadIdx.x & 31, grp = threadIdx.x >> 5;
    const int j = blockIdx.x * 32 + lane;
    float M = -INFINITY, S = 0.f;
    if (j < n) {
        for (int c = grp; c < nchunks; c += kMergeLanes) M = fmaxf(M, part[static_cast<size_t>(c) * part_ld + j].x);
        if (M != -INFINITY)
            for (int c = grp; c < nchunks; c += kMergeLanes) {
                const float2 ps = part[static_cast<size_t>(c) * part_ld + j];
                if (ps.x != -INFINITY) S += ps.y * ex2(ps.x - M);
            }
    }
    red[grp][lane] = make_float2(M, S);
    __syncthreads();
    if (grp == 0 && j < n) {
        float Mt = -INFINITY;
#pragma unroll
        for (int g = 0; g < kMergeLanes; ++g) Mt = fmaxf(Mt, red[g][lane].x);
        float St = 0.f;
        if (Mt != -INFINITY) {
#pragma unroll
            for (int g = 0; g < kMergeLanes; ++g) {
                const float2 ps = red[g][lane];
                if (ps.x != -INFINITY) St += ps.y * ex2(ps.x - Mt);
            }
        }
        b_buf[n_pad + j] = -(Mt + log2f(St)) * kLn2;  // slot of sweep -1 (partials are in base-2 units)
        logcs[j] = 0.f;
    }
}

struct FrameArgs {
    int stream16;      // 1 if a reduced-precision phase exists
    int warmup;        // first reduced-precision sweep index (the absorb sweep)
    int every;         // reabsorb period
    int polish;        // polish sweeps requested
};

// Index of the snapshot that defines the frame of sweep t (or -1 for FP32).
__device__ int frame_snapshot(const FrameArgs& f, int t) {
    if (!f.stream16 || t < f.warmup) return -1;
    return ((t - f.warmup) / f.every) & 1;
}

// Move the final main-phase duals into the FP32 frame and open the polish phase.
__global__ void polish_begin_kernel(SolveState* st, float* a, float* b_buf, long long n_pad, float* logcs,
                                    const float* a_snap, const float* b_snap, int n, FrameArgs f) {
    const int fin = st->final_it;
    const int snap = frame_snapshot(f, fin);
    float* b = b_buf + (fin & 1) * n_pad;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        if (snap >= 0) {
            b[j] += b_snap[snap * n_pad + j];
            a[j] += a_snap[snap * n_pad + j];
        }
        logcs[j] = 0.f;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        st->done = 0;
        st->it = fin + 1;
        st->max_it = fin + 1 + f.polish;
        st->check = 0;
        st->omega = 1.0;
        // the polish sweep's column step is zero (logcs cleared above), so the
        // previous row normaliser is a safe reference: fast path, with the
        // per-row fallback to the exact path when a row sum leaves its range
        st->exact_next = 0;
    }
}

// Final duals (FP32 frame) and the record.
__global__ void solve_end_kernel(const SolveState* st, const float* a, const float* b_buf, long long n_pad,
                                 const float* a_snap, const float* b_snap, int n, FrameArgs f, float* u_out,
                                 float* v_out, fugal_solve_record* rec) {
    const int fin = st->final_it;
    const bool polished = st->check == 0;
    const int snap = polished ? -1 : frame_snapshot(f, fin);
    const float* b = b_buf + (fin & 1) * n_pad;
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        u_out[j] = a[j] + (snap >= 0 ? a_snap[snap * n_pad + j] : 0.f);
        v_out[j] = b[j] + (snap >= 0 ? b_snap[snap * n_pad + j] : 0.f);
    }
    if (rec != nullptr && blockIdx.x == 0) {
        for (int k = threadIdx.x; k < FUGAL_MAX_RECORDED_ERRORS; k += blockDim.x) rec->errors[k] = st->errors[k];
        if (threadIdx.x == 0) {
            rec->iteration_count = st->main_final_it + 1;
            rec->n_errors = min(st->main_n_err, FUGAL_MAX_RECORDED_ERRORS);
            rec->status = st->status;
            rec->polish_count = st->polish_count;
            rec->last_error = st->main_last_err;
            rec->polish_error = st->polish_err;
        }
    }
}

// ------------------------------------------------------------------- host

namespace {

struct SweepPlan {
    int threads;
    int kpt;
    int R;
    int cluster;
    int slice_w;
    int clusters;       // number of clusters in the grid
    int rows_per_cluster;
    int rows_pad;
    int stages;
    size_t smem;
};

int elem_size(int dt) { return dt == FUGAL_F32 ? 4 : 2; }

using KernelFn = void (*)(const SweepArgs);

// mbarrier try_wait suspend-time hint for the sweep's waits, in ns
// (FUGAL_SUSPEND_NS overrides the default).
unsigned suspend_hint() {
    const char* e = getenv("FUGAL_SUSPEND_NS");
    if (e == nullptr) return kSuspendHintNs;
    const long v = atol(e);
    return static_cast<unsigned>(v < 0 ? 0 : (v > 1000000 ? 1000000 : v));
}

// Launch shapes: (threads per CTA, columns per thread).  Rows per batch are
// 32 / columns-per-thread, so a thread always holds 32 exponentials.
constexpr int rows_per_batch(int kpt) { return 32 / kpt; }

using KernelFn = void (*)(const SweepArgs);

template <typename T, int THREADS, int KPT, bool ABSORB, typename TOUT>
KernelFn pick_kernel() {
    return sweep_kernel<T, THREADS, KPT, rows_per_batch(KPT), ABSORB, TOUT>;
}

// kind: 0 = plain sweep over dtype dt, 1 = absorb (fp32 -> bf16), 2 = absorb (fp32 -> fp16)
template <int THREADS, int KPT>
KernelFn kernel_for(int dt, int kind) {
    if (kind == 1) return pick_kernel<float, THREADS, KPT, true, __nv_bfloat16>();
    if (kind == 2) return pick_kernel<float, THREADS, KPT, true, __half>();
    if (dt == FUGAL_BF16) return pick_kernel<__nv_bfloat16, THREADS, KPT, false, float>();
    if (dt == FUGAL_F16) return pick_kernel<__half, THREADS, KPT, false, float>();
    return pick_kernel<float, THREADS, KPT, false, float>();
}

KernelFn kernel_for(int threads, int kpt, int dt, int kind) {
    if (threads == 128) return kpt == 16 ? kernel_for<128, 16>(dt, kind) : kernel_for<128, 32>(dt, kind);
    return kpt == 16 ? kernel_for<256, 16>(dt, kind) : kernel_for<256, 32>(dt, kind);
}

int header_for(int threads, int R) {
    if (threads == 128) return R == 2 ? header_bytes_v3<128, 2>() : header_bytes_v3<128, 1>();
    return R == 2 ? header_bytes_v3<256, 2>() : header_bytes_v3<256, 1>();
}

int max_smem_optin() {
    int dev = 0, v = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev) != cudaSuccess || v <= 0)
        v = 227 * 1024;
    return v;
}

// Column slice per CTA (threads x columns per thread): 8192 (256 x 32) by
// default above 4096 columns; the environment variable FUGAL_SWEEP_SLICE=4096
// selects 256 x 16 (twice the cluster size, two rows per batch) instead.
int slice_choice() {
    const char* e = getenv("FUGAL_SWEEP_SLICE");
    return (e && atoi(e) == 4096) ? 4096 : 8192;
}

// Launch shape for n columns: threads per CTA, columns per thread, CTAs per
// cluster (the smallest power of two covering n).
fugal_status plan_shape(int64_t n, int& threads, int& kpt, int& cluster) {
    // FUGAL_SWEEP_SHAPE="threads,kpt" (threads 128 or 256, kpt 16 or 32) overrides the choice
    const char* shape = getenv("FUGAL_SWEEP_SHAPE");
    int st = 0, sk = 0;
    if (shape != nullptr && sscanf(shape, "%d,%d", &st, &sk) == 2 && (st == 128 || st == 256) &&
        (sk == 16 || sk == 32)) {
        threads = st; kpt = sk;
    } else if (n <= 2048) {
        threads = 128; kpt = 16;
    } else if (n <= 4096) {
        threads = 128; kpt = 32;
    } else if (slice_choice() == 4096) {
        threads = 256; kpt = 16;
    } else {
        threads = 256; kpt = 32;
    }
    const int slice = threads * kpt;
    cluster = 1;
    while (static_cast<int64_t>(cluster) * slice < n) cluster <<= 1;
    if (cluster > kMaxCluster)
        return fail(FUGAL_BAD_SHAPE, "sinkhorn: n = %lld exceeds the supported maximum %d", (long long)n,
                    kMaxCluster * slice);
    return FUGAL_OK;
}

// Dynamic shared memory per CTA kept near 100 KB (with the whole L1 carved out as
// shared memory) so two CTAs (of up to 256 threads) share an SM and hide each
// other's exchange latency; at 104 KB and above the cluster occupancy query
// already settles on one CTA per SM.
constexpr int kSmemTarget = 100 * 1024;

fugal_status make_plan(int64_t n, int dt, int kind, SweepPlan& pl, bool query_occupancy) {
    FUGAL_TRY(plan_shape(n, pl.threads, pl.kpt, pl.cluster));
    const int es = (kind != 0) ? 4 : elem_size(dt);
    pl.R = rows_per_batch(pl.kpt);
    pl.slice_w = pl.threads * pl.kpt;
    const size_t stage_bytes = static_cast<size_t>(pl.R) * pl.slice_w * es;
    const int sms = sm_count();
    const int ctas_per_sm = 2;
    // clusters the grid is expected to hold; the row-dual staging is sized from it
    int est = std::max(1, (sms * ctas_per_sm / pl.cluster) * 3 / 4);
    KernelFn fn = kernel_for(pl.threads, pl.kpt, dt, kind);
    for (int attempt = 0; attempt < 3; ++attempt) {
        pl.rows_pad = static_cast<int>(((n + est - 1) / est + 31) / 32 * 32);
        const size_t fixed = header_for(pl.threads, pl.R) + static_cast<size_t>(pl.slice_w) * 4 +
                             static_cast<size_t>(pl.rows_pad) * 4;
        const int budget = kSmemTarget;
        int stages = static_cast<int>((budget - static_cast<int64_t>(fixed)) / static_cast<int64_t>(stage_bytes));
        stages = std::min(stages, kMaxStages);
        if (stages < 2) stages = std::min(2, static_cast<int>((max_smem_optin() - static_cast<int64_t>(fixed)) /
                                                               static_cast<int64_t>(stage_bytes)));
        if (stages < 1) return fail(FUGAL_BAD_SHAPE, "sinkhorn: no shared-memory stage fits");
        pl.stages = stages;
        pl.smem = fixed + stages * stage_bytes;
        int clusters = sms * 4;  // upper bound for workspace sizing
        if (query_occupancy) {
            FUGAL_TRY(cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pl.smem),
                                 "sinkhorn: set dynamic shared memory"));
            // all of the unified L1 / shared memory as shared memory, so two CTAs fit per SM
            FUGAL_TRY(cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                                      cudaSharedmemCarveoutMaxShared),
                                 "sinkhorn: shared memory carveout"));
            if (pl.cluster > 8)
                FUGAL_TRY(cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeNonPortableClusterSizeAllowed, 1),
                                     "sinkhorn: allow cluster size 16"));
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            cfg.gridDim = dim3(pl.cluster, 1, 1);
            cfg.blockDim = dim3(pl.threads, 1, 1);
            cfg.dynamicSmemBytes = pl.smem;
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = pl.cluster;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int active = 0;
            FUGAL_TRY(cuda_check(cudaOccupancyMaxActiveClusters(&active, fn, &cfg), "sinkhorn: occupancy query"));
            if (active <= 0)
                return fail(FUGAL_UNSUPPORTED, "sinkhorn: cluster of %d CTAs cannot be scheduled", pl.cluster);
            clusters = active;
        }
        const int max_useful = static_cast<int>((n + pl.R - 1) / pl.R);
        clusters = std::max(1, std::min(clusters, max_useful));
        pl.clusters = clusters;
        pl.rows_per_cluster = static_cast<int>((n + clusters - 1) / clusters);
        if (pl.rows_per_cluster <= pl.rows_pad) return FUGAL_OK;
        est = clusters;  // fewer clusters than estimated: size the staging for them and re-plan
    }
    return fail(FUGAL_UNSUPPORTED, "sinkhorn: could not fit the row-dual staging for n = %lld", (long long)n);
}

// Row-owned 16-bit sweep plan (row_sweep_kernel): used for 16-bit sweeps when
// the padded row fits 32768 columns; FUGAL_ROW_SWEEP=0 selects the cluster
// kernel instead.
struct RowPlan {
    bool use = false;
    bool bt = true;
    int poly = 0;
    int cl = 1;      // CTAs per row block (a cluster when 2)
    int groups = 0;  // row blocks (rows of column partials)
    int threads = 512;
    int ept = 0;
    int ctas = 0;
    int rows_per_cta = 0;
    int stages = 0;
    size_t smem = 0;
    KernelFn fn = nullptr;
};

using RowKernelFn = void (*)(const RowArgs);

template <typename T, bool BT, int POLY>
RowKernelFn row_kernel_typed(int ept, int cl) {
    if (cl == 2) return row_sweep_kernel<T, 64, 512, BT, POLY, (BT ? 2 : 1)>;
    return ept == 16 ? row_sweep_kernel<T, 16, 512, BT, POLY, 1>
                     : (ept == 32 ? row_sweep_kernel<T, 32, 512, BT, POLY, 1> : row_sweep_kernel<T, 64, 512, BT, POLY, 1>);
}

template <typename T>
RowKernelFn row_kernel_dt(int ept, bool bt, int poly, int cl) {
    if (!bt) return row_kernel_typed<T, false, 0>(ept, 1);
    switch (poly) {
        case 4: return row_kernel_typed<T, true, 4>(ept, cl);
        case 8: return row_kernel_typed<T, true, 8>(ept, cl);
        default: return row_kernel_typed<T, true, 0>(ept, cl);
    }
}

RowKernelFn row_kernel_for(int dt, int ept, int threads, bool bt, int poly, int cl) {
    (void)threads;
    return dt == FUGAL_BF16 ? row_kernel_dt<__nv_bfloat16>(ept, bt, poly, cl)
                            : row_kernel_dt<__half>(ept, bt, poly, cl);
}

// Share of the row sweep's fast-path exponentials evaluated on the FMA pipe:
// one pair in 8 by default (0.479 -> 0.472 ms per sweep at n = 32768; one in 4
// was slower, 0.489 ms); FUGAL_ROW_POLY=4 or 0 (all on MUFU) overrides.
int row_poly() {
    const char* e = getenv("FUGAL_ROW_POLY");
    const int v = e != nullptr ? atoi(e) : 8;
    return (v == 4 || v == 8) ? v : 0;
}

// Failure-detection test hooks of the row sweep, read from the environment at
// each solve: FUGAL_TEST_WAIT_LIMIT_NS (limit of every bounded wait; unset: 2 s)
// and FUGAL_TEST_FAULT_ROW (a local row of CTA 0 whose copy is armed for 16
// bytes that never arrive, so the waits on it run out; unset: none).
unsigned long long test_wait_limit_ns() {
    const char* e = getenv("FUGAL_TEST_WAIT_LIMIT_NS");
    return e != nullptr ? strtoull(e, nullptr, 10) : 0ull;
}
int test_fault_row() {
    const char* e = getenv("FUGAL_TEST_FAULT_ROW");
    return e != nullptr ? atoi(e) : -1;
}

// Column duals of the row sweep in TMEM (default) or shared memory
// (FUGAL_ROW_DUALS_SMEM=1).
bool row_duals_in_tmem() {
    const char* e = getenv("FUGAL_ROW_DUALS_SMEM");
    return !(e != nullptr && atoi(e) != 0);
}

// Threads per row-sweep CTA: 512.  (A 1024-thread CTA halves the columns per
// thread; at n = 16384 and 32768 the extra per-row reduction and barrier cost
// made it slower.)
int row_threads_for(int64_t) { return 512; }

fugal_status make_row_plan(int64_t n, int dt, int64_t n_pad, RowPlan& rp, bool set_attributes) {
    rp = RowPlan{};
    if (dt == FUGAL_F32) return FUGAL_OK;
    const char* e = getenv("FUGAL_ROW_SWEEP");
    if (e != nullptr && atoi(e) == 0) return FUGAL_OK;
    rp.bt = row_duals_in_tmem();
    // rows up to 32768 columns: one CTA; up to 65536: a cluster of two (duals in TMEM)
    if (n_pad > (rp.bt ? 65536 : 32768)) return FUGAL_OK;
    rp.threads = row_threads_for(n_pad);
    rp.cl = n_pad > 32768 ? 2 : 1;
    const int64_t per_cta = (n_pad + rp.cl - 1) / rp.cl;
    rp.ept = static_cast<int>((per_cta + rp.threads * 16 - 1) / (rp.threads * 16)) * 16;  // 16, 32 or 64
    if (rp.ept == 48) rp.ept = 64;
    const size_t stage_bytes = static_cast<size_t>(rp.threads) * std::min(rp.ept, kRowSeg / rp.threads) * 2;
    rp.poly = rp.bt ? row_poly() : 0;
    // column duals of every covered column, unless they live in TMEM
    const size_t fixed = rp.bt ? 0 : static_cast<size_t>(rp.threads) * rp.ept * 4;
    const int64_t room = static_cast<int64_t>(max_smem_optin()) - 1024 - static_cast<int64_t>(fixed);
    rp.stages = static_cast<int>(std::min<int64_t>(kMaxStages, room / static_cast<int64_t>(stage_bytes)));
    if (rp.stages < 2) return FUGAL_OK;
    rp.smem = fixed + rp.stages * stage_bytes;
    int groups = static_cast<int>(std::min<int64_t>(sm_count() / rp.cl, n));
    RowKernelFn fn = row_kernel_for(dt, rp.ept, rp.threads, rp.bt, rp.poly, rp.cl);
    if (set_attributes) {
        FUGAL_TRY(cuda_check(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rp.smem),
                             "sinkhorn: row sweep shared memory"));
        if (rp.cl > 1) {
            cudaLaunchConfig_t cfg = {};
            cudaLaunchAttribute attr[1];
            cfg.gridDim = dim3(rp.cl, 1, 1);
            cfg.blockDim = dim3(rp.threads, 1, 1);
            cfg.dynamicSmemBytes = rp.smem;
            attr[0].id = cudaLaunchAttributeClusterDimension;
            attr[0].val.clusterDim.x = rp.cl;
            attr[0].val.clusterDim.y = 1;
            attr[0].val.clusterDim.z = 1;
            cfg.attrs = attr;
            cfg.numAttrs = 1;
            int active = 0;
            FUGAL_TRY(cuda_check(cudaOccupancyMaxActiveClusters(&active, fn, &cfg), "sinkhorn: row cluster occupancy"));
            if (active <= 0) return FUGAL_OK;  // no two-CTA cluster fits: the cluster sweep takes over
            groups = static_cast<int>(std::min<int64_t>(active, n));
        }
    }
    rp.rows_per_cta = static_cast<int>((n + groups - 1) / groups);
    rp.groups = static_cast<int>((n + rp.rows_per_cta - 1) / rp.rows_per_cta);
    rp.ctas = rp.groups * rp.cl;
    rp.use = true;
    return FUGAL_OK;
}

constexpr int kColThreads = 256;

int colpass_chunks(int64_t n) {
    const int col_blocks = static_cast<int>((n + kColThreads * 4 - 1) / (kColThreads * 4));
    int chunks = std::max(1, (sm_count() * 8) / std::max(1, col_blocks));
    chunks = std::min<int64_t>(chunks, std::max<int64_t>(1, n / 16));
    return chunks;
}

struct Workspace {
    SolveState* st;
    float* b_buf;     // [2][n_pad]
    float* logcs;     // [n_pad]
    float* a;         // [n_pad]
    float* a_snap;    // [2][n_pad]
    float* b_snap;    // [2][n_pad]
    float* partials;  // [max(sweep clusters, 2*column chunks)][n_pad]
    long long n_pad;
    size_t bytes;
};

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

Workspace layout(int64_t n, char* base, int partial_rows) {
    Workspace w{};
    w.n_pad = static_cast<long long>(align_up(static_cast<size_t>(n), 64));
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off = align_up(off + bytes, 256);
        return p;
    };
    w.st = reinterpret_cast<SolveState*>(take(sizeof(SolveState)));
    w.b_buf = reinterpret_cast<float*>(take(2 * w.n_pad * 4));
    w.logcs = reinterpret_cast<float*>(take(w.n_pad * 4));
    w.a = reinterpret_cast<float*>(take(w.n_pad * 4));
    w.a_snap = reinterpret_cast<float*>(take(2 * w.n_pad * 4));
    w.b_snap = reinterpret_cast<float*>(take(2 * w.n_pad * 4));
    w.partials = reinterpret_cast<float*>(take(static_cast<size_t>(partial_rows) * w.n_pad * 4));
    w.bytes = off;
    return w;
}

int partial_rows_bound(int64_t n) {
    return std::max(sm_count() * 4, 2 * colpass_chunks(n));
}

fugal_status launch_sweep(const SweepPlan& pl, KernelFn fn, const SweepArgs& args, cudaStream_t stream,
                          int family) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    cfg.gridDim = dim3(pl.clusters * pl.cluster, 1, 1);
    cfg.blockDim = dim3(pl.threads, 1, 1);
    cfg.dynamicSmemBytes = pl.smem;
    cfg.stream = stream;
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = pl.cluster;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    LaunchScope scope(family, stream);
    return cuda_check(cudaLaunchKernelEx(&cfg, fn, args), "sinkhorn: sweep launch");
}

// Ring of pinned host words receiving the device "done" flag at each poll;
// every solve takes two fresh slots so a late copy of an earlier solve on
// another stream cannot be mistaken for this one's.
constexpr int kPinnedSlots = 64;
// The host reads the flag copied at an evaluation point kPollLag sweeps later:
// the stream still holds that many sweeps of work while the host waits, and at
// most kPollLag sweeps (which return at once) are launched after convergence.
constexpr int kPollLag = 2;
thread_local int* g_pinned_ring = nullptr;
thread_local int g_pinned_next = 0;

}  // namespace

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_sinkhorn_workspace_size(int64_t n, int stream_dtype, size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_workspace_size: null output");
    if (n <= 0) return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_workspace_size: n must be positive");
    if (stream_dtype < FUGAL_F32 || stream_dtype > FUGAL_F16)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_workspace_size: bad stream dtype");
    int threads, kpt, cluster;
    FUGAL_TRY(plan_shape(n, threads, kpt, cluster));
    *bytes = layout(n, nullptr, partial_rows_bound(n)).bytes;
    return FUGAL_OK;
}

extern "C" fugal_status fugal_sinkhorn_plan_info(int64_t n, int stream_dtype, int32_t* info) {
    if (info == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_plan_info: null output");
    if (stream_dtype < FUGAL_F32 || stream_dtype > FUGAL_F16)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_plan_info: bad stream dtype");
    RowPlan rp;
    FUGAL_TRY(make_row_plan(n, stream_dtype, static_cast<int64_t>(align_up(static_cast<size_t>(n), 64)), rp, false));
    if (rp.use) {  // row-owned sweep: one CTA per SM, no cluster
        info[0] = rp.threads;
        info[1] = rp.cl;
        info[2] = rp.groups;
        info[3] = rp.stages;
        info[4] = static_cast<int32_t>(rp.smem);
        info[5] = 1;
        return FUGAL_OK;
    }
    SweepPlan pl;
    FUGAL_TRY(make_plan(n, stream_dtype, 0, pl, true));
    info[0] = pl.threads;
    info[1] = pl.cluster;
    info[2] = pl.clusters;
    info[3] = pl.stages;
    info[4] = static_cast<int32_t>(pl.smem);
    info[5] = pl.R;
    return FUGAL_OK;
}

extern "C" fugal_status fugal_sinkhorn_solve(const fugal_solve_params* prm, void* workspace, size_t workspace_bytes,
                                             fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (prm == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_solve: null params");
    const fugal_solve_params& p = *prm;
    const int64_t n = p.n;
    if (n <= 0) return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_solve: n must be positive");
    if (p.cost32 == nullptr || p.u_out == nullptr || p.v_out == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_solve: null pointer argument");
    if (p.stream_dtype < FUGAL_F32 || p.stream_dtype > FUGAL_F16)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_solve: bad stream dtype");
    const bool use16 = p.stream_dtype != FUGAL_F32;
    if (use16 && p.cost16 == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_solve: cost16 is null");
    if (p.max_iterations <= 0 || p.eval_freq <= 0)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_solve: max_iterations and eval_freq must be positive");
    if (p.ld32 < n || (p.ld32 % 4) != 0 || !aligned16(p.cost32))
        return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_solve: cost32 needs ld >= n, ld %% 4 == 0, 16-byte base");
    if (p.ld32 >= (1ll << 32) || (use16 && p.ld16 >= (1ll << 32)))
        return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_solve: leading dimensions must be below 2^32");
    if (use16 && (p.ld16 < n || (p.ld16 % 8) != 0 || !aligned16(p.cost16)))
        return fail(FUGAL_BAD_SHAPE, "fugal_sinkhorn_solve: cost16 needs ld >= n, ld %% 8 == 0, 16-byte base");
    if (use16 && (p.fp32_warmup_sweeps < 0 || p.reabsorb_every <= 0 || p.polish_sweeps < 0))
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_solve: bad reduced-precision schedule");
    if (p.column_partials != nullptr &&
        (p.column_partial_chunks <= 0 || p.column_partial_ld < n ||
         (reinterpret_cast<uintptr_t>(p.column_partials) & 7u) != 0))
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sinkhorn_solve: column partials need chunks > 0, ld >= n, 8-byte base");

    const int prow = partial_rows_bound(n);
    Workspace w = layout(n, static_cast<char*>(workspace), prow);
    if (workspace_bytes < w.bytes)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_sinkhorn_solve: workspace %zu < %zu bytes", workspace_bytes,
                    w.bytes);

    SweepPlan plan32{}, plan16{}, plan_abs{};
    RowPlan rowplan;
    FUGAL_TRY(make_plan(n, FUGAL_F32, 0, plan32, true));
    if (use16) FUGAL_TRY(make_row_plan(n, p.stream_dtype, w.n_pad, rowplan, true));
    if (use16) {
        if (!rowplan.use) FUGAL_TRY(make_plan(n, p.stream_dtype, 0, plan16, true));
        FUGAL_TRY(make_plan(n, FUGAL_F32, p.stream_dtype == FUGAL_BF16 ? 1 : 2, plan_abs, true));
    }
    if (plan32.clusters > prow || (use16 && (plan16.clusters > prow || plan_abs.clusters > prow)) ||
        rowplan.groups > prow)
        return fail(FUGAL_UNSUPPORTED, "fugal_sinkhorn_solve: more clusters than partial rows");

    FrameArgs frame{use16 ? 1 : 0, use16 ? p.fp32_warmup_sweeps : 0, use16 ? p.reabsorb_every : 1,
                    use16 ? p.polish_sweeps : 0};

    // ---- iteration 0, column update: v_0 = -LSE_i(cost32_ij + a_i), a = 0, from
    //      the caller's column partials (written with the cost) or a pass over cost32
    FUGAL_TRY(cuda_check(cudaMemsetAsync(w.a, 0, w.n_pad * 4, stream), "sinkhorn: clear row duals"));
    const float2* part = reinterpret_cast<const float2*>(w.partials);
    int chunks = colpass_chunks(n);
    long long part_ld = w.n_pad;
    if (p.column_partials != nullptr) {
        part = reinterpret_cast<const float2*>(p.column_partials);
        chunks = p.column_partial_chunks;
        part_ld = p.column_partial_ld;
    } else {
        const int rows_per_chunk = static_cast<int>((n + chunks - 1) / chunks);
        dim3 grid(static_cast<unsigned>((n + kColThreads * 4 - 1) / (kColThreads * 4)), chunks);
        LaunchScope scope(FUGAL_KERNEL_COLUMN_PASS, stream);
        column_pass_kernel<<<grid, kColThreads, 0, stream>>>(p.cost32, p.ld32, static_cast<int>(n), w.a,
                                                              rows_per_chunk, reinterpret_cast<float2*>(w.partials),
                                                              w.n_pad);
        FUGAL_TRY(launch_check("sinkhorn: column pass"));
    }
    const int fin_blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4 * sm_count()));
    {
        InitArgs ia{p.max_iterations, p.eval_freq, p.momentum_start < 0 ? -1 : p.momentum_start, p.threshold};
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        column_merge_kernel<<<static_cast<unsigned>((n + 31) / 32), 256, 0, stream>>>(
            part, chunks, part_ld, w.n_pad, static_cast<int>(n), w.b_buf, w.logcs, w.st, ia);
        FUGAL_TRY(launch_check("sinkhorn: column merge"));
    }

    auto sweep_args = [&](const SweepPlan& pl, const void* L, long long ld, const float* b_off,
                          const float* a_off) {
        SweepArgs a{};
        a.L = L;
        a.ld = ld;
        a.n = static_cast<int>(n);
        const int es = (L == p.cost32) ? 4 : elem_size(p.stream_dtype);
        const int V = 16 / es;
        a.n_copy = static_cast<int>((n + V - 1) / V * V);
        a.slice_w = pl.slice_w;
        a.rows_per_cluster = pl.rows_per_cluster;
        a.rows_pad = pl.rows_pad;
        a.suspend_ns = suspend_hint();
        a.stages = pl.stages;
        a.b_buf = w.b_buf;
        a.b_buf_w = w.b_buf;
        a.b_off = b_off;
        a.logcs = w.logcs;
        a.a = w.a;
        a.a_off = a_off;
        a.partials = w.partials;
        a.n_pad = w.n_pad;
        a.st = w.st;
        return a;
    };
    const int fin_grid = static_cast<int>((n + kFinCols - 1) / kFinCols);
    auto finalize = [&](int nparts) -> fugal_status {
        LaunchScope scope(FUGAL_KERNEL_FINALIZE, stream);
        finalize_kernel<<<fin_grid, kFinThreads, 0, stream>>>(w.partials, nparts, w.n_pad, static_cast<int>(n),
                                                              w.logcs, w.st);
        return launch_check("sinkhorn: finalize");
    };

    // ---- main phase: sweeps t = 0 .. max_iterations-1, polled at evaluation points
    if (g_pinned_ring == nullptr) {
        void* ptr = nullptr;
        FUGAL_TRY(cuda_check(cudaHostAlloc(&ptr, kPinnedSlots * sizeof(int), cudaHostAllocPortable),
                             "sinkhorn: pinned flags"));
        g_pinned_ring = static_cast<int*>(ptr);
    }
    int* g_pinned_done = g_pinned_ring + g_pinned_next;
    g_pinned_next = (g_pinned_next + 2) % kPinnedSlots;
    cudaEvent_t ev[2] = {nullptr, nullptr};
    FUGAL_TRY(cuda_check(cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming), "sinkhorn: event"));
    FUGAL_TRY(cuda_check(cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming), "sinkhorn: event"));
    auto destroy = [&]() {
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
    };
    int slot = 0;
    int poll_slot = -1, poll_t = 0;  // the copy of `done` in flight, issued after sweep poll_t
    fugal_status status = FUGAL_OK;
    auto read_poll = [&](bool& stop) -> fugal_status {
        const fugal_status s = cuda_check(cudaEventSynchronize(ev[poll_slot]), "sinkhorn: poll wait");
        timing_poll();
        stop = s == FUGAL_OK && g_pinned_done[poll_slot] != 0;
        poll_slot = -1;
        return s;
    };
    for (int t = 0; t < p.max_iterations && status == FUGAL_OK; ++t) {
        const int snap_idx = (!use16 || t < p.fp32_warmup_sweeps) ? -1 : ((t - p.fp32_warmup_sweeps) / p.reabsorb_every);
        const bool absorb = use16 && t >= p.fp32_warmup_sweeps && (t - p.fp32_warmup_sweeps) % p.reabsorb_every == 0;
        if (!use16 || t < p.fp32_warmup_sweeps) {
            SweepArgs a = sweep_args(plan32, p.cost32, p.ld32, nullptr, nullptr);
            status = launch_sweep(plan32, kernel_for(plan32.threads, plan32.kpt, FUGAL_F32, 0), a, stream, FUGAL_KERNEL_SWEEP_F32);
            if (status == FUGAL_OK) status = finalize(plan32.clusters);
        } else if (absorb) {
            // reads cost32 in the FP32 frame (offsets of the previous snapshot if any), writes snapshot snap_idx
            const float* b_off = snap_idx > 0 ? w.b_snap + ((snap_idx - 1) & 1) * w.n_pad : nullptr;
            const float* a_off = snap_idx > 0 ? w.a_snap + ((snap_idx - 1) & 1) * w.n_pad : nullptr;
            SweepArgs a = sweep_args(plan_abs, p.cost32, p.ld32, b_off, a_off);
            a.out16 = p.cost16;
            a.ld16 = p.ld16;
            a.a_snap = w.a_snap + (snap_idx & 1) * w.n_pad;
            a.b_snap = w.b_snap + (snap_idx & 1) * w.n_pad;
            status = launch_sweep(plan_abs, kernel_for(plan_abs.threads, plan_abs.kpt, FUGAL_F32, p.stream_dtype == FUGAL_BF16 ? 1 : 2),
                                  a, stream, FUGAL_KERNEL_ABSORB);
            if (status == FUGAL_OK) status = finalize(plan_abs.clusters);
        } else if (rowplan.use) {
            RowArgs ra{};
            ra.L = p.cost16;
            ra.ld = p.ld16;
            ra.n = static_cast<int>(n);
            ra.n_copy = static_cast<int>((n + 7) / 8 * 8);
            ra.rows_per_cta = rowplan.rows_per_cta;
            ra.stages = rowplan.stages;
            ra.suspend_ns = suspend_hint();
            ra.b_buf = w.b_buf;
            ra.logcs = w.logcs;
            ra.b_buf_w = w.b_buf;
            ra.a = w.a;
            ra.partials = w.partials;
            ra.n_pad = w.n_pad;
            ra.st = w.st;
            ra.wait_limit_ns = test_wait_limit_ns();
            ra.fault_row = test_fault_row();
            {
                LaunchScope scope(FUGAL_KERNEL_SWEEP, stream);
                RowKernelFn fn = row_kernel_for(p.stream_dtype, rowplan.ept, rowplan.threads, rowplan.bt,
                                                rowplan.poly, rowplan.cl);
                if (rowplan.cl == 1) {
                    fn<<<rowplan.ctas, rowplan.threads, rowplan.smem, stream>>>(ra);
                    status = launch_check("sinkhorn: row sweep");
                } else {
                    cudaLaunchConfig_t cfg = {};
                    cudaLaunchAttribute attr[1];
                    cfg.gridDim = dim3(rowplan.ctas, 1, 1);
                    cfg.blockDim = dim3(rowplan.threads, 1, 1);
                    cfg.dynamicSmemBytes = rowplan.smem;
                    cfg.stream = stream;
                    attr[0].id = cudaLaunchAttributeClusterDimension;
                    attr[0].val.clusterDim.x = rowplan.cl;
                    attr[0].val.clusterDim.y = 1;
                    attr[0].val.clusterDim.z = 1;
                    cfg.attrs = attr;
                    cfg.numAttrs = 1;
                    status = cuda_check(cudaLaunchKernelEx(&cfg, fn, ra), "sinkhorn: row sweep launch");
                }
            }
            if (status == FUGAL_OK) status = finalize(rowplan.groups);
        } else {
            SweepArgs a = sweep_args(plan16, p.cost16, p.ld16, nullptr, nullptr);
            status = launch_sweep(plan16, kernel_for(plan16.threads, plan16.kpt, p.stream_dtype, 0), a, stream, FUGAL_KERNEL_SWEEP);
            if (status == FUGAL_OK) status = finalize(plan16.clusters);
        }
        if (status != FUGAL_OK) break;
        bool stop = false;
        if (poll_slot >= 0 && t - poll_t >= kPollLag) {
            status = read_poll(stop);
            if (status != FUGAL_OK || stop) break;
        }
        const bool eval_point = (t % p.eval_freq == 0 && t != 0);
        if (eval_point) {
            if (poll_slot >= 0) {  // eval_freq < kPollLag: settle the older poll first
                status = read_poll(stop);
                if (status != FUGAL_OK || stop) break;
            }
            slot ^= 1;
            status = cuda_check(cudaMemcpyAsync(&g_pinned_done[slot], &w.st->done, sizeof(int),
                                                cudaMemcpyDeviceToHost, stream),
                                "sinkhorn: poll copy");
            if (status == FUGAL_OK) status = cuda_check(cudaEventRecord(ev[slot], stream), "sinkhorn: poll event");
            poll_slot = slot;
            poll_t = t;
        }
    }
    if (status != FUGAL_OK) {
        destroy();
        return status;
    }

    // ---- polish: FP32 sweeps on cost32 after a reduced-precision phase
    const int nblk = fin_blocks;
    if (use16 && p.polish_sweeps > 0) {
        {
            LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
            polish_begin_kernel<<<nblk, 256, 0, stream>>>(w.st, w.a, w.b_buf, w.n_pad, w.logcs, w.a_snap, w.b_snap,
                                                          static_cast<int>(n), frame);
            status = launch_check("sinkhorn: polish begin");
        }
        for (int k = 0; k < p.polish_sweeps && status == FUGAL_OK; ++k) {
            SweepArgs a = sweep_args(plan32, p.cost32, p.ld32, nullptr, nullptr);
            status = launch_sweep(plan32, kernel_for(plan32.threads, plan32.kpt, FUGAL_F32, 0), a, stream, FUGAL_KERNEL_SWEEP_F32);
            if (status == FUGAL_OK) status = finalize(plan32.clusters);
        }
    }
    if (status == FUGAL_OK) {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        solve_end_kernel<<<nblk, 256, 0, stream>>>(w.st, w.a, w.b_buf, w.n_pad, w.a_snap, w.b_snap,
                                                   static_cast<int>(n), frame, p.u_out, p.v_out,
                                                   static_cast<fugal_solve_record*>(p.record));
        status = launch_check("sinkhorn: solve end");
    }
    destroy();
    return status;
}
