// hzb_vmb.cu -- VMB aggregation (aggregation_vmb, amg_setup_ua.c:596-736),
// the greedy aggregation of Vanek, Mandel and Brezina on the strength graph,
// with the reference's visiting orders and counters:
//   step 1, rows descending: a row whose strength-graph row has only one
//     entry becomes UNPT; a row whose every neighbour (itself included) is
//     still unvisited (-2) opens an aggregate with up to max_aggregation - 1
//     of its other neighbours, in row order;
//   step 2, rows descending, on the step-1 map: an unvisited row joins the
//     first neighbour's step-1 aggregate (row order) that has fewer than
//     max_aggregation members (sizes counted as the step goes);
//   step 3, while the reference's count of unvisited rows is positive (one
//     ascending pass always ends it: the count never exceeds the true number),
//     an unvisited row opens an aggregate with its unvisited neighbours.
// Each step is sequential in the reference; here one warp walks the rows
// (lanes cover a row's entries and chunks of rows) with the state in global
// memory, __syncwarp between rows.  No aggregate after step 1 is the
// reference's ERROR_AMG_COARSEING: *nagg = 0 and the caller stops coarsening.
#include "hzb_setup.cuh"

namespace hzb {

namespace {
constexpr unsigned FULL = 0xffffffffu;
constexpr int UNVISITED = -2;

__global__ void k_vmb_fill(int n, int *agg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        agg[i] = UNVISITED;
}

// out[0] = aggregates, out[1] = the reference's num_left
__global__ void __launch_bounds__(32)
k_vmb_step1(int n, const int *__restrict__ ia, const int *__restrict__ ja, int max_agg,
            int *agg_, int *out) {
    volatile int *agg = agg_;
    const int lane = threadIdx.x;
    int na = 0, left = n;
    for (int i = n - 1; i >= 0; --i) {
        const int b0 = ia[i], b1 = ia[i + 1];
        if (b1 - b0 == 1) {
            if (lane == 0) agg[i] = UNPT;
            --left;
            __syncwarp();
            continue;
        }
        bool taken = false;
        for (int base = b0; base < b1; base += 32) {
            const int p = base + lane;
            const bool t = p < b1 && agg[ja[p]] >= UNPT;
            if (__any_sync(FULL, t)) { taken = true; break; }
        }
        if (!taken) {
            if (lane == 0) agg[i] = na;
            int count = 1;
            for (int base = b0; base < b1 && count < max_agg; base += 32) {
                const int p = base + lane;
                const int c = p < b1 ? ja[p] : -1;
                const bool e = p < b1 && c != i;
                const unsigned m = __ballot_sync(FULL, e);
                const int rank = __popc(m & ((1u << lane) - 1u));
                if (e && count + rank < max_agg) agg[c] = na;
                count += min(__popc(m), max_agg - count);
            }
            left -= count;
            ++na;
        }
        __syncwarp();
    }
    if (lane == 0) {
        out[0] = na;
        out[1] = left;
    }
}

// the step-1 map (temp_C) and its aggregate sizes
__global__ void k_vmb_count(int n, const int *__restrict__ agg, int *temp, int *cnt) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int a = agg[i];
        temp[i] = a;
        if (a >= 0) atomicAdd(cnt + a, 1);
    }
}

__global__ void __launch_bounds__(32)
k_vmb_step2(int n, const int *__restrict__ ia, const int *__restrict__ ja, int max_agg,
            int *agg_, const int *__restrict__ temp, int *cnt_, int *out) {
    volatile int *agg = agg_;
    volatile int *cnt = cnt_;
    const int lane = threadIdx.x;
    int left = out[1];
    for (int base = n - 1; base >= 0; base -= 32) {
        const int i = base - lane;   // lane 0 holds the highest row of the chunk
        unsigned m = __ballot_sync(FULL, i >= 0 && agg[i] < UNPT);
        while (m) {
            const int r = base - (__ffs(m) - 1);
            m &= m - 1;
            const int b0 = ia[r], b1 = ia[r + 1];
            for (int pb = b0; pb < b1; pb += 32) {
                const int p = pb + lane;
                int a = UNPT;
                bool ok = false;
                if (p < b1) {
                    a = temp[ja[p]];
                    ok = a > UNPT && cnt[a] < max_agg;
                }
                const unsigned mm = __ballot_sync(FULL, ok);
                if (mm) {
                    const int aa = __shfl_sync(FULL, a, __ffs(mm) - 1);
                    if (lane == 0) {
                        agg[r] = aa;
                        cnt[aa] = cnt[aa] + 1;
                    }
                    --left;
                    break;
                }
            }
            __syncwarp();
        }
    }
    if (lane == 0) out[1] = left;
}

__global__ void __launch_bounds__(32)
k_vmb_step3(int n, const int *__restrict__ ia, const int *__restrict__ ja, int max_agg,
            int *agg_, int *out) {
    volatile int *agg = agg_;
    const int lane = threadIdx.x;
    if (out[1] <= 0) return;
    int na = out[0], left = out[1];
    for (int base = 0; base < n; base += 32) {
        const int i = base + lane;
        unsigned m = __ballot_sync(FULL, i < n && agg[i] < UNPT);
        while (m) {
            const int r = base + __ffs(m) - 1;
            m &= m - 1;
            // a row opened earlier in this chunk may have taken r
            if (lane == 0 && agg[r] < UNPT) {
                agg[r] = na;
                int count = 1;
                --left;
                for (int p = ia[r]; p < ia[r + 1]; ++p) {
                    const int c = ja[p];
                    if (c != r && agg[c] < UNPT && count < max_agg) {
                        agg[c] = na;
                        --left;
                        ++count;
                    }
                }
                ++na;
            }
            __syncwarp();
        }
    }
    if (lane == 0) {
        out[0] = na;
        out[1] = left;
    }
}

// rows left without an aggregate get an empty row of P (form_tentative_p)
__global__ void k_vmb_final(int n, int *agg) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (agg[i] < 0) agg[i] = UNPT;
}
}  // namespace

int vmb_aggregate(int n, const int *nia, const int *nja, int max_agg, int *agg, int *nagg,
                  int *work, cudaStream_t s) {
    *nagg = 0;
    if (n <= 0) return SUCCESS;
    int *temp = work, *cnt = work + n, *out = nullptr;
    HZB_TRY(dalloc(&out, 2));
    k_vmb_fill<<<grid_for(n), 256, 0, s>>>(n, agg);
    k_vmb_step1<<<1, 32, 0, s>>>(n, nia, nja, max_agg, agg, out);
    count_launch(2);
    int h[2] = {0, 0};
    cudaError_t e = cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e != cudaSuccess) {
        dfree(out);
        set_error(e, __FILE__, __LINE__);
        return ERROR_SOLVER_MISC;
    }
    if (h[0] < MIN_CDOF) {   // the reference's ERROR_AMG_COARSEING after step 1
        dfree(out);
        return SUCCESS;
    }
    e = cudaMemsetAsync(cnt, 0, sizeof(int) * n, s);
    if (e == cudaSuccess) {
        k_vmb_count<<<grid_for(n), 256, 0, s>>>(n, agg, temp, cnt);
        k_vmb_step2<<<1, 32, 0, s>>>(n, nia, nja, max_agg, agg, temp, cnt, out);
        k_vmb_step3<<<1, 32, 0, s>>>(n, nia, nja, max_agg, agg, out);
        k_vmb_final<<<grid_for(n), 256, 0, s>>>(n, agg);
        count_launch(4);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(h, out, sizeof(h), cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    dfree(out);
    if (e != cudaSuccess) {
        set_error(e, __FILE__, __LINE__);
        return ERROR_SOLVER_MISC;
    }
    *nagg = h[0];
    return SUCCESS;
}

}  // namespace hzb
