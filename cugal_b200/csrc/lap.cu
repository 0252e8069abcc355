// Greedy rounding of the quasi-permutation (cugal/greedy_lap.py:7-85).
//
// The reference processes rows one at a time with a torch launch and a host
// read each (`row *= taken; m = row.argmax(); taken[m] = 0; m.item()`), i.e. n
// dependent round trips.  The result is fully determined by the row order and
// the rule "column = first index of the maximum of row * taken", so it can be
// reproduced exactly with far less work on the critical path:
//
//  1. candidates: one pass over P keeps, per row, its top-K columns in the
//     total order (value desc, index asc) plus the row maximum / arg-maximum.
//  2. order: rows by descending maximum, ties by lower row index (a stable
//     sort; the reference's argsort is unstable, see below), by counting ranks.
//  3. walk: one CTA walks the rows in order.  The first not-yet-taken candidate
//     of a row is its exact answer whenever its value is > 0 (every column
//     outside the top-K ranks below it, and taken columns read as 0).
//     Otherwise -- all K candidates taken, or the best free value is 0 -- the
//     CTA scans the full row under the taken mask (same rule as the reference).
//  4. mutate (optional): P[r][j] *= 0 for every column taken before row r's
//     turn, which is exactly how the reference leaves P behind (Q4).
//
// Tie order note: torch's argsort(descending=True) is not stable, so for rows
// with identical maxima the reference's order is unspecified; this kernel uses
// the stable order (ties by row index), the same as the oracle.
#include <cuda_runtime.h>

#include <algorithm>
#include <climits>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kMaxCand = 16;
constexpr int kCandThreads = 256;

// (value desc, index asc) total order: true if (va, ia) ranks before (vb, ib).
__device__ __forceinline__ bool better(float va, int ia, float vb, int ib) {
    return va > vb || (va == vb && ia < ib);
}

template <int K>
__global__ void __launch_bounds__(kCandThreads) candidates_kernel(const float* __restrict__ P, long long ldp, int n,
                                                                  int* cand_idx, float* cand_val, float* row_max,
                                                                  int* row_arg) {
    __shared__ int wt[kCandThreads / 32];
    __shared__ float wv[kCandThreads / 32];
    __shared__ int wi[kCandThreads / 32];
    __shared__ int win_thread;
    const int r = blockIdx.x;
    const float* row = P + static_cast<size_t>(r) * ldp;
    float tv[K];
    int ti[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
        tv[k] = -INFINITY;
        ti[k] = INT_MAX;
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x) {
        const float x = row[j];
        if (better(x, j, tv[K - 1], ti[K - 1])) {
            // insert keeping tv/ti sorted by the total order
            float cv = x;
            int ci = j;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                if (better(cv, ci, tv[k], ti[k])) {
                    const float sv = tv[k];
                    const int si = ti[k];
                    tv[k] = cv;
                    ti[k] = ci;
                    cv = sv;
                    ci = si;
                }
            }
        }
    }
    // K rounds of a block-wide arg-best over the threads' list heads.
    int head = 0;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = 0; k < K; ++k) {
        float v = -INFINITY;
        int idx = INT_MAX;
#pragma unroll
        for (int q = 0; q < K; ++q)
            if (q == head) {
                v = tv[q];
                idx = ti[q];
            }
        float bv = v;
        int bi = idx;
        int bt = threadIdx.x;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
            const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
            const int ot = __shfl_xor_sync(0xffffffffu, bt, o);
            if (better(ov, oi, bv, bi)) {
                bv = ov;
                bi = oi;
                bt = ot;
            }
        }
        if (lane == 0) {
            wv[warp] = bv;
            wi[warp] = bi;
            wt[warp] = bt;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            float b = wv[0];
            int bidx = wi[0], bthr = wt[0];
            for (int w = 1; w < kCandThreads / 32; ++w)
                if (better(wv[w], wi[w], b, bidx)) {
                    b = wv[w];
                    bidx = wi[w];
                    bthr = wt[w];
                }
            cand_val[static_cast<size_t>(r) * K + k] = b;
            cand_idx[static_cast<size_t>(r) * K + k] = bidx;
            if (k == 0) {
                row_max[r] = b;
                row_arg[r] = bidx;
            }
            win_thread = bthr;
        }
        __syncthreads();
        if (threadIdx.x == win_thread) ++head;
        __syncthreads();
    }
}

// rank of row i = #rows with larger maximum + #earlier rows with an equal maximum.
__global__ void __launch_bounds__(256) rank_rows_kernel(const float* __restrict__ key, int n, int* order) {
    __shared__ float tile[1024];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    // NaN keys rank as -inf so the ranks always form a permutation
    auto clean = [](float x) { return isnan(x) ? -INFINITY : x; };
    const float ki = i < n ? clean(key[i]) : 0.f;
    int rank = 0;
    for (int base = 0; base < n; base += 1024) {
        for (int q = threadIdx.x; q < 1024; q += blockDim.x) tile[q] = base + q < n ? clean(key[base + q]) : -INFINITY;
        __syncthreads();
        const int lim = min(1024, n - base);
        if (i < n) {
            for (int q = 0; q < lim; ++q) {
                const float kj = tile[q];
                const int j = base + q;
                rank += (kj > ki || (kj == ki && j < i)) ? 1 : 0;
            }
        }
        __syncthreads();
    }
    if (i < n) order[rank] = i;
}

__global__ void iota_kernel(int* order, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) order[i] = i;
}
// Caller-given order; an entry outside [0, n) is replaced by -1 and skipped by the walk.
__global__ void copy_order_kernel(const long long* src, int* order, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const long long r = src[i];
        order[i] = (r >= 0 && r < n) ? static_cast<int>(r) : -1;
    }
}

constexpr int kWalkThreads = 1024;
constexpr int kWalkBatch = 256;
constexpr int kMaxWalkN = 1 << 18;  // taken mask lives in shared memory (32 KB)

struct WalkArgs {
    const float* P;
    long long ldp;
    int n;
    int K;
    const int* order;
    const int* cand_idx;
    const float* cand_val;
    const float* row_max;
    const int* row_arg;
    int parallel_phase;     // PARALLEL_GREEDY: rows with max > 0.5 take their arg-max first
    long long* columns;
    int* pos;               // position of each row in the walk (-1: parallel phase)
    int* owner_pos;         // first position at which each column was taken (INT_MAX: never)
};

__device__ __forceinline__ bool is_taken(const unsigned int* t, int j) { return (t[j >> 5] >> (j & 31)) & 1u; }

// Dynamic shared memory: taken mask [ceil(n/32)] words, then the batch's
// candidates [kWalkBatch][K] indices and values.
__global__ void __launch_bounds__(kWalkThreads) walk_kernel(const WalkArgs a) {
    extern __shared__ __align__(16) unsigned char walk_smem[];
    __shared__ int ord_s[kWalkBatch];
    __shared__ int resolved_s;
    __shared__ float rv[kWalkThreads / 32];
    __shared__ int ri[kWalkThreads / 32];
    const int n = a.n, K = a.K;
    const int words = (n + 31) >> 5;
    unsigned int* taken = reinterpret_cast<unsigned int*>(walk_smem);
    int* cidx = reinterpret_cast<int*>(taken + ((words + 3) & ~3));
    float* cval = reinterpret_cast<float*>(cidx + kWalkBatch * K);
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int q = tid; q < words; q += blockDim.x) taken[q] = 0u;
    __syncthreads();

    int p0 = 0;
    if (a.parallel_phase) {
        // the order is by descending maximum, so rows with max > 0.5 form a prefix
        if (tid == 0) {
            int q = 0;
            while (q < n && a.order[q] >= 0 && a.row_max[a.order[q]] > 0.5f) ++q;
            resolved_s = q;
        }
        __syncthreads();
        p0 = resolved_s;
        for (int q = tid; q < p0; q += blockDim.x) {
            const int r = a.order[q];
            const int c = a.row_arg[r];
            a.columns[r] = c;
            a.pos[r] = -1;
            atomicOr(&taken[c >> 5], 1u << (c & 31));
            atomicMin(&a.owner_pos[c], -1);
        }
        __syncthreads();
    }

    for (int p = p0; p < n; p += kWalkBatch) {
        const int batch = min(kWalkBatch, n - p);
        for (int q = tid; q < batch; q += blockDim.x) ord_s[q] = a.order[p + q];
        __syncthreads();
        for (int q = tid; q < batch * K; q += blockDim.x) {
            const int r = ord_s[q / K];
            cidx[q] = r >= 0 ? a.cand_idx[static_cast<size_t>(r) * K + (q % K)] : -1;
            cval[q] = r >= 0 ? a.cand_val[static_cast<size_t>(r) * K + (q % K)] : 0.f;
        }
        __syncthreads();
        int q = 0;
        while (true) {
            if (tid == 0) {
                while (q < batch) {
                    const int r = ord_s[q];
                    if (r < 0) {  // invalid caller-given row: skipped
                        ++q;
                        continue;
                    }
                    int c = -1;
                    float v = 0.f;
                    for (int k = 0; k < K; ++k) {
                        const int ck = cidx[q * K + k];
                        if (ck < 0 || ck >= n) break;  // row shorter than K
                        if (!is_taken(taken, ck)) {
                            c = ck;
                            v = cval[q * K + k];
                            break;
                        }
                    }
                    if (c < 0 || !(v > 0.f)) break;  // needs the full-row rule
                    a.columns[r] = c;
                    a.pos[r] = p + q;
                    taken[c >> 5] |= 1u << (c & 31);
                    if (a.owner_pos[c] == INT_MAX) a.owner_pos[c] = p + q;
                    ++q;
                }
                resolved_s = q;
            }
            __syncthreads();
            q = resolved_s;
            __syncthreads();  // every thread has read resolved_s before it is written again
            if (q >= batch) break;
            // full-row rule for row ord_s[q]: first index of the maximum of row * taken
            const int r = ord_s[q];
            const float* row = a.P + static_cast<size_t>(r) * a.ldp;
            float bv = -INFINITY;
            int bi = INT_MAX;
            for (int j = tid; j < n; j += blockDim.x) {
                const float x = is_taken(taken, j) ? row[j] * 0.0f : row[j];
                if (better(x, j, bv, bi)) {
                    bv = x;
                    bi = j;
                }
            }
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const float ov = __shfl_xor_sync(0xffffffffu, bv, o);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
                if (better(ov, oi, bv, bi)) {
                    bv = ov;
                    bi = oi;
                }
            }
            if (lane == 0) {
                rv[warp] = bv;
                ri[warp] = bi;
            }
            __syncthreads();
            if (tid == 0) {
                float b = rv[0];
                int c = ri[0];
                for (int w = 1; w < kWalkThreads / 32; ++w)
                    if (better(rv[w], ri[w], b, c)) {
                        b = rv[w];
                        c = ri[w];
                    }
                if (c < 0 || c >= n) c = 0;
                a.columns[r] = c;
                a.pos[r] = p + q;
                taken[c >> 5] |= 1u << (c & 31);
                if (a.owner_pos[c] == INT_MAX) a.owner_pos[c] = p + q;
            }
            __syncthreads();  // taken mask and rv/ri settled before the next round
            ++q;
        }
        __syncthreads();
    }
}

size_t walk_smem_bytes(int64_t n, int K) {
    const size_t words = ((n + 31) / 32 + 3) / 4 * 4;
    return words * 4 + static_cast<size_t>(kWalkBatch) * K * 8;
}

// P[r][j] *= 0 for columns taken before row r was processed (rows of the walk only).
__global__ void mutate_kernel(float* P, long long ldp, int n, const int* pos, const int* owner_pos) {
    const int r = blockIdx.x;
    const int pr = pos[r];
    if (pr < 0) return;
    float* row = P + static_cast<size_t>(r) * ldp;
    for (int j = blockIdx.y * blockDim.x + threadIdx.x; j < n; j += gridDim.y * blockDim.x)
        if (owner_pos[j] < pr) row[j] = row[j] * 0.0f;
}

__global__ void init_walk_kernel(int* owner_pos, int n) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) owner_pos[i] = INT_MAX;
}

struct LapWs {
    int* cand_idx;
    float* cand_val;
    float* row_max;
    int* row_arg;
    int* order;
    int* pos;
    int* owner_pos;
    size_t bytes;
};

LapWs lap_layout(int64_t n, int K, char* base) {
    LapWs w{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off = (off + bytes + 255) / 256 * 256;
        return p;
    };
    w.cand_idx = reinterpret_cast<int*>(take(static_cast<size_t>(n) * K * 4));
    w.cand_val = reinterpret_cast<float*>(take(static_cast<size_t>(n) * K * 4));
    w.row_max = reinterpret_cast<float*>(take(n * 4));
    w.row_arg = reinterpret_cast<int*>(take(n * 4));
    w.order = reinterpret_cast<int*>(take(n * 4));
    w.pos = reinterpret_cast<int*>(take(n * 4));
    w.owner_pos = reinterpret_cast<int*>(take(n * 4));
    w.bytes = off;
    return w;
}

// ---------------------------------------------------------------------------
// MORE_RAND (cugal/greedy_lap.py:34-48): rows in a caller-given random order;
// row r is masked by the free columns (row *= taken), and its column is the
// first index j whose running sum of the masked row reaches x = total * u_k
// (u_k the k-th draw of Python's random.random(), so that
// random.uniform(0, total) = total * u_k).  One CTA walks the rows: a pass over
// the row forms 32-column chunk sums (FP64, each an inclusive warp scan), a
// block scan over them finds the chunk where the running sum reaches x, and one
// warp scans that chunk again with the same operations for the column.  The
// free-column mask is a bit set in shared memory.
constexpr int kSampleThreads = 1024;
constexpr int kMaxSampleN = 1 << 19;

__device__ __forceinline__ double warp_inclusive_scan(double v) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const double t = __shfl_up_sync(0xffffffffu, v, o);
        if (lane >= o) v += t;
    }
    return v;
}

__global__ void __launch_bounds__(kSampleThreads) sampled_walk_kernel(float* P, long long ldp, int n,
                                                                      const long long* order, const double* uniforms,
                                                                      int mutate, long long* cols) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int nch = (n + 31) / 32;
    double* csum = reinterpret_cast<double*>(smem);        // [nch] chunk sums of the masked row
    unsigned* taken = reinterpret_cast<unsigned*>(csum + nch);  // [nch] bit (j % 32) of word j / 32
    __shared__ double wscan[32];
    __shared__ double s_before, s_total;
    __shared__ int s_chunk;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    for (int c = tid; c < nch; c += kSampleThreads) taken[c] = 0u;
    const int per = (nch + kSampleThreads - 1) / kSampleThreads;
    const int c0 = min(nch, tid * per), c1 = min(nch, c0 + per);
    __syncthreads();
    for (int k = 0; k < n; ++k) {
        const long long r = order[k];
        float* row = P + static_cast<size_t>(r) * ldp;
        // chunk sums of row * free (the masked entries written back when mutating)
        for (int c = warp; c < nch; c += kSampleThreads / 32) {
            const int j = c * 32 + lane;
            float v = 0.f;
            if (j < n) {
                v = row[j];
                if ((taken[c] >> lane) & 1u) {
                    v = v * 0.f;
                    if (mutate) row[j] = v;
                }
            }
            const double incl = warp_inclusive_scan(static_cast<double>(v));
            if (lane == 31) csum[c] = incl;
        }
        __syncthreads();
        // block exclusive scan of the per-thread chunk ranges
        double ts = 0.0;
        for (int c = c0; c < c1; ++c) ts += csum[c];
        const double incl = warp_inclusive_scan(ts);
        if (lane == 31) wscan[warp] = incl;
        if (tid == 0) s_chunk = INT_MAX;
        __syncthreads();
        if (warp == 0) {
            const double wv = wscan[lane];
            const double wi = warp_inclusive_scan(wv);
            wscan[lane] = wi - wv;
        }
        __syncthreads();
        const double before = wscan[warp] + (incl - ts);
        // the total is the running sum as the last thread forms it, so some chunk reaches x
        double cum = before;
        for (int c = c0; c < c1; ++c) cum += csum[c];
        if (tid == kSampleThreads - 1) s_total = cum;
        __syncthreads();
        const double x = s_total * uniforms[k];
        cum = before;
        int found = INT_MAX;
        for (int c = c0; c < c1; ++c) {
            const double nxt = cum + csum[c];
            if (x <= nxt) {
                found = c;
                break;
            }
            cum = nxt;
        }
        if (found != INT_MAX) atomicMin(&s_chunk, found);
        __syncthreads();
        if (found != INT_MAX && found == s_chunk) s_before = cum;
        __syncthreads();
        if (warp == 0) {
            const int c = s_chunk == INT_MAX ? nch - 1 : s_chunk;
            const int j = c * 32 + lane;
            float v = 0.f;
            if (j < n) {
                v = row[j];
                if ((taken[c] >> lane) & 1u) v = v * 0.f;
            }
            const double run = s_before + warp_inclusive_scan(static_cast<double>(v));
            const unsigned hit = __ballot_sync(0xffffffffu, j < n && x <= run);
            const int m = hit ? c * 32 + __ffs(hit) - 1 : min(n - 1, c * 32 + 31);
            if (lane == 0) {
                taken[m / 32] |= 1u << (m % 32);
                cols[r] = m;
            }
        }
        __syncthreads();
    }
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_sampled_lap(float* P, int64_t ldp, int64_t n, const int64_t* order,
                                          const double* uniforms, int mutate, int64_t* columns_out,
                                          fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    if (P == nullptr || order == nullptr || uniforms == nullptr || columns_out == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_sampled_lap: null argument");
    if (n <= 0 || n > kMaxSampleN) return fail(FUGAL_BAD_SHAPE, "fugal_sampled_lap: n must be in [1, %d]", kMaxSampleN);
    if (ldp < n) return fail(FUGAL_BAD_SHAPE, "fugal_sampled_lap: ldp < n");
    const size_t nch = static_cast<size_t>((n + 31) / 32);
    const size_t smem = nch * (sizeof(double) + sizeof(unsigned));
    FUGAL_TRY(cuda_check(cudaFuncSetAttribute(sampled_walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              static_cast<int>(smem)),
                         "fugal_sampled_lap: shared memory"));
    LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
    sampled_walk_kernel<<<1, kSampleThreads, smem, stream>>>(P, ldp, static_cast<int>(n),
                                                             reinterpret_cast<const long long*>(order), uniforms,
                                                             mutate, reinterpret_cast<long long*>(columns_out));
    return launch_check("fugal_sampled_lap");
}

extern "C" fugal_status fugal_greedy_lap_workspace_size(int64_t n, int candidates, size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_greedy_lap_workspace_size: null output");
    if (n <= 0 || n > kMaxWalkN)
        return fail(FUGAL_BAD_SHAPE, "fugal_greedy_lap_workspace_size: n must be in [1, %d]", kMaxWalkN);
    if (candidates < 1 || candidates > kMaxCand)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_greedy_lap_workspace_size: candidates must be in [1, %d]", kMaxCand);
    *bytes = lap_layout(n, candidates, nullptr).bytes;
    return FUGAL_OK;
}

extern "C" fugal_status fugal_greedy_lap(float* P, int64_t ldp, int64_t n, int method, const int64_t* order,
                                         int candidates, int mutate, int64_t* columns_out, void* workspace,
                                         size_t workspace_bytes, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    size_t need = 0;
    FUGAL_TRY(fugal_greedy_lap_workspace_size(n, candidates, &need));
    if (P == nullptr || columns_out == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_greedy_lap: null argument");
    if (ldp < n) return fail(FUGAL_BAD_SHAPE, "fugal_greedy_lap: ldp < n");
    if (method < FUGAL_LAP_GREEDY || method > FUGAL_LAP_ORDERED)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_greedy_lap: bad method %d", method);
    if (method == FUGAL_LAP_ORDERED && order == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_greedy_lap: ORDERED needs an order");
    if (workspace_bytes < need)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_greedy_lap: workspace %zu < %zu", workspace_bytes, need);
    LapWs w = lap_layout(n, candidates, static_cast<char*>(workspace));
    const int nn = static_cast<int>(n);
    const int K = candidates;
    const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4 * sm_count()));
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        init_walk_kernel<<<blocks, 256, 0, stream>>>(w.owner_pos, nn);
        FUGAL_TRY(launch_check("fugal_greedy_lap: init"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
#define FUGAL_CAND(KK)                                                                                    \
    case KK:                                                                                              \
        candidates_kernel<KK><<<nn, kCandThreads, 0, stream>>>(P, ldp, nn, w.cand_idx, w.cand_val, w.row_max, \
                                                               w.row_arg);                                \
        break;
        switch (K) {
            FUGAL_CAND(1) FUGAL_CAND(2) FUGAL_CAND(4) FUGAL_CAND(8) FUGAL_CAND(16)
            default:
                return fail(FUGAL_BAD_ARGUMENT, "fugal_greedy_lap: candidates must be 1, 2, 4, 8 or 16");
        }
#undef FUGAL_CAND
        FUGAL_TRY(launch_check("fugal_greedy_lap: candidates"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        if (method == FUGAL_LAP_GREEDY)
            iota_kernel<<<blocks, 256, 0, stream>>>(w.order, nn);
        else if (method == FUGAL_LAP_ORDERED)
            copy_order_kernel<<<blocks, 256, 0, stream>>>(reinterpret_cast<const long long*>(order), w.order, nn);
        else
            rank_rows_kernel<<<(nn + 255) / 256, 256, 0, stream>>>(w.row_max, nn, w.order);
        FUGAL_TRY(launch_check("fugal_greedy_lap: order"));
    }
    {
        WalkArgs a{P, ldp, nn, K, w.order, w.cand_idx, w.cand_val, w.row_max, w.row_arg,
                   method == FUGAL_LAP_PARALLEL_GREEDY ? 1 : 0, reinterpret_cast<long long*>(columns_out), w.pos,
                   w.owner_pos};
        const size_t smem = walk_smem_bytes(n, K);
        FUGAL_TRY(cuda_check(cudaFuncSetAttribute(walk_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  static_cast<int>(smem)),
                             "fugal_greedy_lap: walk shared memory"));
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        walk_kernel<<<1, kWalkThreads, smem, stream>>>(a);
        FUGAL_TRY(launch_check("fugal_greedy_lap: walk"));
    }
    if (mutate) {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        dim3 grid(static_cast<unsigned>(nn), static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 64)));
        mutate_kernel<<<grid, 256, 0, stream>>>(P, ldp, nn, w.pos, w.owner_pos);
        FUGAL_TRY(launch_check("fugal_greedy_lap: mutate"));
    }
    return FUGAL_OK;
}
