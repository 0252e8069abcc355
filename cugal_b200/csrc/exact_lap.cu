// Exact linear assignment on the device, with the same mapping as
// scipy.optimize.linear_sum_assignment (the reference's HungarianMethod.SCIPY,
// cugal/pred.py:151-158; scipy 1.18.1 here).
//
// scipy solves the assignment with the shortest-augmenting-path method of
// D. F. Crouse, "On implementing 2D rectangular assignment algorithms", IEEE
// TAES 52(4), 2016: rows are added one at a time; for each, a Dijkstra search
// over reduced costs  minVal + c_ij - u_i - v_j  finds the cheapest path to a
// free column, then the duals u, v are updated and the path is augmented.  For
// the mapping to be identical to scipy's -- including which optimum it returns
// when several exist -- this kernel reproduces scipy's choices exactly:
//
//   * maximize: c = -P (the FP32 P converted to double first);
//   * the candidate columns are kept in a list that starts in descending column
//     order and loses the selected column by "swap with the last entry";
//   * each step selects the minimum shortest-path cost; among equal minima the
//     first one in list order, unless a later equal one is an unassigned
//     column, in which case the last such unassigned column;
//   * all arithmetic in double, in scipy's operation order (additions and
//     subtractions only, each rounded on its own).
//
// One CTA runs the outer loop over rows; each Dijkstra step scans the
// remaining columns with all its threads and reduces (cost, tie priority) with
// warp shuffles.  The list order is restored after every row from an undo log,
// and shortest-path costs are invalidated by a row stamp, so the per-row
// bookkeeping costs O(path length), not O(n).  A cap on the total number of
// Dijkstra steps bounds the run time; hitting it is reported in the status word.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>

#include "fugal_common.cuh"
#include "fugal_host.h"

namespace fugal {

constexpr int kExactThreads = 1024;

struct ExactWs {
    double* u;
    double* v;
    double* spc;    // shortest-path cost per column (valid when stamp == current row)
    int* stamp;
    int* path;
    int* col4row;
    int* row4col;
    int* remaining;
    int* sr_list;   // rows reached in the current search
    int* sc_list;   // columns reached (= removed from the list) in the current search
    int* undo_idx;  // list positions overwritten by those removals
    int* bad;       // count of invalid entries (NaN, or -inf cost)
    size_t bytes;
};

ExactWs exact_layout(int64_t n, char* base) {
    ExactWs w{};
    size_t off = 0;
    auto take = [&](size_t bytes) {
        char* p = base ? base + off : nullptr;
        off = (off + bytes + 255) / 256 * 256;
        return p;
    };
    w.u = reinterpret_cast<double*>(take(n * 8));
    w.v = reinterpret_cast<double*>(take(n * 8));
    w.spc = reinterpret_cast<double*>(take(n * 8));
    w.stamp = reinterpret_cast<int*>(take(n * 4));
    w.path = reinterpret_cast<int*>(take(n * 4));
    w.col4row = reinterpret_cast<int*>(take(n * 4));
    w.row4col = reinterpret_cast<int*>(take(n * 4));
    w.remaining = reinterpret_cast<int*>(take(n * 4));
    w.sr_list = reinterpret_cast<int*>(take(n * 4));
    w.sc_list = reinterpret_cast<int*>(take(n * 4));
    w.undo_idx = reinterpret_cast<int*>(take(n * 4));
    w.bad = reinterpret_cast<int*>(take(4));
    w.bytes = off;
    return w;
}

// Invalid entries for scipy: NaN anywhere, or a cost of -inf (P = +inf when maximizing).
__global__ void exact_check_kernel(const float* __restrict__ P, long long ldp, int n, int maximize, int* bad) {
    int cnt = 0;
    for (int r = blockIdx.y; r < n; r += gridDim.y) {
        const float* row = P + static_cast<size_t>(r) * ldp;
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
            const float c = maximize ? -row[j] : row[j];
            if (c != c || c == -INFINITY) ++cnt;
        }
    }
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(bad, cnt);
}

__global__ void exact_init_kernel(ExactWs w, int n) {
    for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
        w.u[j] = 0.0;
        w.v[j] = 0.0;
        w.stamp[j] = -1;
        w.path[j] = -1;
        w.col4row[j] = -1;
        w.row4col[j] = -1;
        w.remaining[j] = n - 1 - j;  // descending column order, as scipy fills it
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) *w.bad = 0;
}

// Selection key of a column in one Dijkstra step: smaller cost wins; among equal
// costs an unassigned column beats an assigned one, unassigned columns later in
// the list beat earlier ones and assigned columns earlier in the list beat later
// ones.  `prio` encodes that tie order (larger wins) and the list position.
struct Pick {
    double cost;
    int prio;
};
constexpr int kPrioBase = 1 << 30;
__device__ __forceinline__ int pick_prio(int pos, bool unassigned) {
    return unassigned ? kPrioBase + pos : kPrioBase - 1 - pos;
}
__device__ __forceinline__ int prio_pos(int prio) { return prio >= kPrioBase ? prio - kPrioBase : kPrioBase - 1 - prio; }
__device__ __forceinline__ Pick pick_better(Pick a, Pick b) {
    return (a.cost < b.cost || (a.cost == b.cost && a.prio > b.prio)) ? a : b;
}
__device__ __forceinline__ Pick pick_warp(Pick a) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        Pick b;
        b.cost = __shfl_xor_sync(0xffffffffu, a.cost, o);
        b.prio = __shfl_xor_sync(0xffffffffu, a.prio, o);
        a = pick_better(a, b);
    }
    return a;
}

__global__ void __launch_bounds__(kExactThreads) exact_lap_kernel(const float* __restrict__ P, long long ldp, int n,
                                                                  int maximize, long long max_steps, ExactWs w,
                                                                  long long* columns_out, long long* steps_out,
                                                                  int* status_out) {
    __shared__ Pick warp_best[kExactThreads / 32];
    __shared__ int s_i, s_sink, s_num, s_nsr, s_nsc, s_stop;
    __shared__ double s_min;
    __shared__ long long s_steps;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (*w.bad != 0) {
        if (tid == 0) {
            *status_out = FUGAL_NONFINITE;
            if (steps_out) *steps_out = 0;
        }
        return;
    }
    if (tid == 0) {
        s_steps = 0;
        s_stop = 0;
    }
    for (int cur = 0; cur < n; ++cur) {
        if (tid == 0) {
            s_i = cur;
            s_min = 0.0;
            s_sink = -1;
            s_num = n;
            s_nsr = 1;
            w.sr_list[0] = cur;
            s_nsc = 0;
        }
        __syncthreads();
        // ---- shortest augmenting path from row `cur`
        while (true) {
            const int i = s_i;
            const double min_val = s_min;
            const int num = s_num;
            const double ui = w.u[i];
            const float* prow = P + static_cast<size_t>(i) * ldp;
            Pick best{INFINITY, -1};
            for (int it = tid; it < num; it += kExactThreads) {
                const int j = w.remaining[it];
                const double p = static_cast<double>(prow[j]);
                const double c = maximize ? -p : p;
                const double r = __dsub_rn(__dsub_rn(__dadd_rn(min_val, c), ui), w.v[j]);
                double sp = (w.stamp[j] == cur) ? w.spc[j] : INFINITY;
                if (r < sp) {
                    w.path[j] = i;
                    w.spc[j] = r;
                    w.stamp[j] = cur;
                    sp = r;
                }
                best = pick_better(best, Pick{sp, pick_prio(it, w.row4col[j] < 0)});
            }
            best = pick_warp(best);
            if (lane == 0) warp_best[warp] = best;
            __syncthreads();
            if (warp == 0) {
                Pick b = warp_best[lane];
                b = pick_warp(b);
                if (lane == 0) {
                    const long long steps = ++s_steps;
                    if (b.cost == INFINITY || b.prio < 0) {
                        *status_out = FUGAL_BAD_ARGUMENT;  // infeasible: every remaining cost is +inf
                        s_stop = 1;
                    } else if (steps > max_steps) {
                        *status_out = FUGAL_ITER_LIMIT;
                        s_stop = 1;
                    } else {
                        const int idx = prio_pos(b.prio);
                        const int j = w.remaining[idx];
                        s_min = b.cost;
                        if (w.row4col[j] < 0) {
                            s_sink = j;
                        } else {
                            s_i = w.row4col[j];
                            w.sr_list[s_nsr++] = s_i;
                        }
                        w.undo_idx[s_nsc] = idx;
                        w.sc_list[s_nsc++] = j;
                        w.remaining[idx] = w.remaining[num - 1];
                        s_num = num - 1;
                    }
                }
            }
            __syncthreads();
            if (s_sink >= 0 || s_stop) break;
        }
        if (s_stop) break;
        // ---- duals (scipy: u[cur] += minVal; u[i] += minVal - spc[col4row[i]]; v[j] -= minVal - spc[j])
        const double min_val = s_min;
        for (int k = tid; k < s_nsr; k += kExactThreads) {
            const int i2 = w.sr_list[k];
            if (i2 == cur)
                w.u[i2] = __dadd_rn(w.u[i2], min_val);
            else
                w.u[i2] = __dadd_rn(w.u[i2], __dsub_rn(min_val, w.spc[w.col4row[i2]]));
        }
        for (int k = tid; k < s_nsc; k += kExactThreads) {
            const int j2 = w.sc_list[k];
            w.v[j2] = __dsub_rn(w.v[j2], __dsub_rn(min_val, w.spc[j2]));
        }
        __syncthreads();
        if (tid == 0) {
            // augment along the path
            int j = s_sink;
            while (true) {
                const int i2 = w.path[j];
                w.row4col[j] = i2;
                const int t = w.col4row[i2];
                w.col4row[i2] = j;
                j = t;
                if (i2 == cur) break;
            }
            // restore the candidate list to its state at the start of the row
            for (int k = s_nsc - 1; k >= 0; --k) w.remaining[w.undo_idx[k]] = w.sc_list[k];
        }
        __syncthreads();
    }
    if (s_stop) {
        if (tid == 0 && steps_out) *steps_out = s_steps;
        return;
    }
    for (int r = tid; r < n; r += kExactThreads) columns_out[r] = w.col4row[r];
    if (tid == 0) {
        *status_out = FUGAL_OK;
        if (steps_out) *steps_out = s_steps;
    }
}

}  // namespace fugal

using namespace fugal;

extern "C" fugal_status fugal_exact_lap_workspace_size(int64_t n, size_t* bytes) {
    if (bytes == nullptr) return fail(FUGAL_BAD_ARGUMENT, "fugal_exact_lap_workspace_size: null output");
    if (n <= 0 || n >= (1 << 30)) return fail(FUGAL_BAD_SHAPE, "fugal_exact_lap_workspace_size: bad n");
    *bytes = exact_layout(n, nullptr).bytes;
    return FUGAL_OK;
}

extern "C" fugal_status fugal_exact_lap(const float* P, int64_t ldp, int64_t n, int maximize, int64_t max_steps,
                                        int64_t* columns_out, int64_t* steps_out, int32_t* status_out,
                                        void* workspace, size_t workspace_bytes, fugal_stream_t stream_) {
    cudaStream_t stream = reinterpret_cast<cudaStream_t>(stream_);
    size_t need = 0;
    FUGAL_TRY(fugal_exact_lap_workspace_size(n, &need));
    if (P == nullptr || columns_out == nullptr || status_out == nullptr || workspace == nullptr)
        return fail(FUGAL_BAD_ARGUMENT, "fugal_exact_lap: null argument");
    if (ldp < n) return fail(FUGAL_BAD_SHAPE, "fugal_exact_lap: ldp < n");
    if (max_steps <= 0) return fail(FUGAL_BAD_ARGUMENT, "fugal_exact_lap: max_steps must be positive");
    if (workspace_bytes < need)
        return fail(FUGAL_WORKSPACE_TOO_SMALL, "fugal_exact_lap: workspace %zu < %zu", workspace_bytes, need);
    ExactWs w = exact_layout(n, static_cast<char*>(workspace));
    const int nn = static_cast<int>(n);
    const int blocks = static_cast<int>(std::min<int64_t>((n + 255) / 256, 4 * sm_count()));
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        exact_init_kernel<<<blocks, 256, 0, stream>>>(w, nn);
        FUGAL_TRY(launch_check("fugal_exact_lap: init"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        dim3 grid(static_cast<unsigned>(std::min<int64_t>((n + 255) / 256, 8)),
                  static_cast<unsigned>(std::min<int64_t>(n, 4 * sm_count())));
        exact_check_kernel<<<grid, 256, 0, stream>>>(P, ldp, nn, maximize ? 1 : 0, w.bad);
        FUGAL_TRY(launch_check("fugal_exact_lap: check"));
    }
    {
        LaunchScope scope(FUGAL_KERNEL_OTHER, stream);
        exact_lap_kernel<<<1, kExactThreads, 0, stream>>>(P, ldp, nn, maximize ? 1 : 0, max_steps, w,
                                                          reinterpret_cast<long long*>(columns_out),
                                                          reinterpret_cast<long long*>(steps_out), status_out);
        FUGAL_TRY(launch_check("fugal_exact_lap: solve"));
    }
    return FUGAL_OK;
}
