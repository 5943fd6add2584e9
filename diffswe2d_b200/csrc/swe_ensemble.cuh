// swe_ensemble.cuh -- scheduler of the persistent ensemble kernel, shared by
// the IEEE (swe_step.cu) and tolerance-mode (swe_fast.cu) step kernels.
#pragma once

#include "swe_sweep.cuh"

namespace swe {

// ---------------------------------------------------------------------------
// Persistent ensemble kernel: many independent scenarios of different grid
// sizes, each with its own time step, boundary series and step count, in
// one launch.
//
// Work item = (scenario, phase, tile); phase 2n is stage 1 of step n, phase
// 2n+1 its stage 2.  Each scenario keeps a 64-bit claim word (phase << 32 |
// tiles claimed) and a done counter.  A block claims a tile with one
// atomicAdd on the claim word; when the phase is fully claimed it tries the
// next scenario.  The block that completes a phase's last tile advances the
// scenario (time, step count, next boundary level, cleared reductions) and
// publishes the next phase with atomicExch.  No block ever waits for a
// particular item, so the kernel cannot deadlock; idle polling is bounded
// (__nanosleep back-off, and a time limit without progress given at launch)
// after which the kernel sets an error bit and returns.  State written by other blocks is read through
// L2 (ld.global.cg); writes are fenced before a phase is published.
struct EnsCtl {
    unsigned long long claim;  // phase << 32 | tiles claimed
    unsigned int done;         // tiles finished in the current phase
    unsigned int red[SWE_RED_WORDS];
    float level;               // boundary level of the current step
    int step;                  // steps completed
    int finished;              // 0 running, 1 done, 2 failed
    int tiles, nbx, rows, steps;
    int nseries;
    float dt_last;
    unsigned int status;
    double time;               // simulated time since the start
    double start;
    const float* series_t;
    const float* series_w;
    float* Ua;                 // state buffers: step n reads U[n & 1]
    float* Ub;
    // interval mode (n_out > 0)
    double out_dt, elapsed, tol, cap;
    int n_out, chunk, ngauge, nx;
    float max_dt_cur;          // max_dt of the current step (both modes)
    const float* out_levels;
    const int32_t* gauge_cells;
    float* gauge_out;
    const float* bed;
};

struct EnsGlobal {
    unsigned int finished;  // scenarios done or failed
    unsigned int error;     // bit 1: no progress within the launch's idle limit
    unsigned int progress;  // phases completed, all scenarios
    unsigned int pad[13];
};

// Default idle limit of the persistent kernel: phases complete in
// microseconds to milliseconds, so two seconds without progress anywhere
// means the launch cannot finish.
constexpr unsigned long long EnsStallNsDefault = 2000000000ull;

static __device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

static __device__ float ens_level(const EnsCtl& c) {
    if (c.nseries <= 0) return c.level;
    const float t = (float)(c.start + c.time);
    const float* times = c.series_t;
    const float* levels = c.series_w;
    const int n = c.nseries;
    if (n == 1) return levels[0];
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (times[mid] < t) lo = mid + 1;
        else hi = mid;
    }
    const int idx = min(max(lo, 1), n - 1);
    const float t0 = times[idx - 1], t1 = times[idx];
    const float weight = __fdiv_rn(t - t0, fmaxf(t1 - t0, 1.1920929e-07f));
    return levels[idx - 1] + weight * (levels[idx] - levels[idx - 1]);
}

// Thread 0 of the block that finished the last tile of `phase`.
static __device__ void ens_advance(EnsCtl* c, EnsGlobal* g, unsigned int phase) {
    __threadfence();
    c->done = 0u;
    const unsigned int st = __ldcg(&c->red[2]);
    if ((phase & 1u) == 0u) {  // stage 1 done: stage 2 derives dt from red
        if (st & SWE_S_NONFINITE_STATE) {
            c->status = st;
            c->finished = 2;
            __threadfence();
            atomicAdd(&g->finished, 1u);
            atomicAdd(&g->progress, 1u);
            return;
        }
    } else {  // stage 2 done: the step is complete
        const float dt = __uint_as_float(__ldcg(&c->red[3]));
        if (st & (SWE_S_NONFINITE_DT | SWE_S_NONPOSITIVE_DT)) {
            c->status = st;
            c->finished = 2;
            __threadfence();
            atomicAdd(&g->finished, 1u);
            atomicAdd(&g->progress, 1u);
            return;
        }
        c->time += (double)dt;
        c->dt_last = dt;
        const int done_step = c->step;
        c->step = done_step + 1;
        int fin = 0;
        if (c->n_out > 0) {
            // the interval bookkeeping of swe_run_clock_f32 (solver.py:741-768)
            double el = c->elapsed + (double)dt;
            if (el > c->out_dt && el - c->out_dt <= c->tol) el = c->out_dt;
            if (c->out_dt - el <= c->tol) {
                const float* Unew = (done_step & 1) ? c->Ua : c->Ub;  // this step's output
                for (int q = 0; q < c->ngauge; ++q) {
                    const size_t cell = (size_t)c->gauge_cells[2 * q] * c->nx + c->gauge_cells[2 * q + 1];
                    c->gauge_out[(size_t)c->chunk * c->ngauge + q] = __ldcg(Unew + cell) + c->bed[cell];
                }
                c->chunk += 1;
                el = 0.0;
                if (c->chunk >= c->n_out) fin = 1;
            }
            c->elapsed = el;
            if (!fin && c->step >= c->steps) {
                c->status = SWE_S_STEP_LIMIT;
                fin = 2;
            }
            if (!fin) {
                const double rem = c->out_dt - el;
                c->max_dt_cur = (float)((c->cap > 0.0 && c->cap < rem) ? c->cap : rem);
                c->level = c->out_levels[c->chunk];
            }
        } else {
            if (c->step >= c->steps) fin = 1;
            else c->level = ens_level(*c);
        }
        if (fin) {
            c->finished = fin;
            __threadfence();
            atomicAdd(&g->finished, 1u);
            atomicAdd(&g->progress, 1u);
            return;
        }
        for (int w = 0; w < SWE_RED_WORDS; ++w) c->red[w] = 0u;
    }
    __threadfence();
    atomicExch(&c->claim, (unsigned long long)(phase + 1u) << 32);
    atomicAdd(&g->progress, 1u);
}

// The body of the persistent kernel; T::run<STAGE, FRIC>(args, bx, by, rows)
// computes one tile of one stage in the arithmetic of the including file.
// An idle block gives up (error bit 1) when no scenario has completed a
// phase for stall_ns nanoseconds.
template <int FRIC, class T>
__device__ __forceinline__ void ensemble_body(const StepArgs* __restrict__ args, EnsCtl* ctl, int count,
                                              EnsGlobal* g, unsigned long long stall_ns) {
    __shared__ StepArgs sa;
    __shared__ int s_item[3];
    int rr = (int)(blockIdx.x % (unsigned)count);
    unsigned int seen_progress = 0xffffffffu, backoff = 64;
    unsigned long long seen_at = 0;
    while (true) {
        __syncthreads();  // everyone is done with the previous item's shared data
        if (threadIdx.x == 0) {
            int item = -2, phase = 0, tile = 0;
            for (int k = 0; k < count && item == -2; ++k) {
                const int sidx = (rr + k) % count;
                EnsCtl* c = ctl + sidx;
                if (*(volatile int*)&c->finished) continue;
                // a fully claimed phase is skipped without an atomic (idle
                // blocks would otherwise all bump the last busy claim word)
                if ((unsigned int)*(volatile unsigned long long*)&c->claim >= (unsigned int)c->tiles) continue;
                const unsigned long long old = atomicAdd(&c->claim, 1ull);
                const unsigned int ph = (unsigned int)(old >> 32), cl = (unsigned int)old;
                if (cl < (unsigned int)c->tiles) {
                    item = sidx;
                    phase = (int)ph;
                    tile = (int)cl;
                    rr = sidx;
                }
            }
            if (item == -2) {
                const unsigned int prog = *(volatile unsigned int*)&g->progress;
                const unsigned long long now = global_ns();
                if (*(volatile unsigned int*)&g->finished >= (unsigned int)count ||
                    *(volatile unsigned int*)&g->error) {
                    item = -1;
                } else if (prog != seen_progress) {
                    seen_progress = prog;
                    seen_at = now;
                    __nanosleep(backoff);
                } else if (now - seen_at > stall_ns) {
                    atomicOr(&g->error, 1u);
                    item = -1;
                } else {
                    __nanosleep(backoff);
                    backoff = min(backoff * 2u, 4096u);
                }
            } else {
                backoff = 64;
                __threadfence();
            }
            s_item[0] = item;
            s_item[1] = phase;
            s_item[2] = tile;
        }
        __syncthreads();
        const int sidx = s_item[0];
        if (sidx == -1) return;
        if (sidx == -2) continue;
        const int phase = s_item[1], tile = s_item[2];
        // this scenario's arguments, with the state buffers of this step
        {
            const int* src = reinterpret_cast<const int*>(args + sidx);
            int* dst = reinterpret_cast<int*>(&sa);
            for (int w = threadIdx.x; w < (int)(sizeof(StepArgs) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
        }
        __syncthreads();
        const EnsCtl* c = ctl + sidx;
        const int step = phase >> 1;
        if (threadIdx.x == 0) {
            sa.U = (step & 1) ? c->Ub : c->Ua;
            sa.U_out = (step & 1) ? c->Ua : c->Ub;
            sa.max_dt = __ldcg(&c->max_dt_cur);
        }
        __syncthreads();
        const int nbx = c->nbx, rows = c->rows;
        const int bx = tile % nbx, by = tile / nbx;
        if ((phase & 1) == 0) T::template run<1, 0>(sa, bx, by, rows);
        else T::template run<2, FRIC>(sa, bx, by, rows);
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0) {
            EnsCtl* cw = ctl + sidx;
            const unsigned int d = atomicAdd(&cw->done, 1u);
            if (d + 1u == (unsigned int)cw->tiles) ens_advance(cw, g, (unsigned int)phase);
        }
    }
}

// The tolerance-mode persistent kernel (swe_fast.cu).
int fast_launch_ensemble(int friction, int blocks, const StepArgs* args, EnsCtl* ctl, int count,
                         EnsGlobal* g, unsigned long long stall_ns, cudaStream_t s);

}  // namespace swe
