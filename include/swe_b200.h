/*
 * swe_b200.h -- C ABI of the B200 shallow-water step library
 * (diffswe2d_b200/_lib/libswe_b200.so).
 *
 * Each entry point replaces one function of the DiffSWE2d reference (cited
 * as path:line within that project) on the device path.  Conventions:
 *   - every pointer is a device pointer to contiguous float32 NCHW data
 *     unless stated otherwise; the caller (PyTorch) allocates every buffer
 *     and the library frees nothing; it keeps no pointer to caller memory
 *     across calls (its own state: the per-device address of the static
 *     scratch of swe_step_noalloc_f32 and the tile-height knob);
 *   - "B" is the batch, "ny, nx" the interior grid; fields with a batch of 1
 *     broadcast over the batch (bedB, nB, levelB = 1 or B);
 *   - work is enqueued on `stream` (a cudaStream_t passed as void*);
 *     nothing synchronises the host;
 *   - the return value is SWE_OK or an SWE_E* code; a CUDA launch error is
 *     reported as SWE_ECUDA.
 * Numerical failures found on the device (non-finite state or time step,
 * non-positive time step) are written as SWE_S* bits into a device status
 * word that the caller reads with the step's time step.
 */
#ifndef SWE_B200_H
#define SWE_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Return codes. */
#define SWE_OK 0
#define SWE_EARG 1  /* invalid argument (shape, size, code) */
#define SWE_ECUDA 2 /* CUDA launch or runtime error */

/* Device status bits. */
#define SWE_S_NONFINITE_STATE 1u /* NaN/Inf in the state read by a step */
#define SWE_S_NONFINITE_DT 2u    /* non-finite CFL time step */
#define SWE_S_NONPOSITIVE_DT 4u  /* time step <= 0 */
#define SWE_S_STEP_LIMIT 8u      /* ensemble member in interval mode reached its step cap */

/* Boundary codes (src/boundary.py:11-18). */
#define SWE_BC_TRANSMISSIVE 0
#define SWE_BC_PERIODIC 1
#define SWE_BC_CONSTANT 2
#define SWE_BC_WATER_LEVEL 3
#define SWE_BC_WALL 4
#define SWE_BC_ABSORBING 5

/* Forcing modes for rain / infiltration arguments. */
#define SWE_FORCING_NONE 0
#define SWE_FORCING_SCALAR 1 /* one value (device pointer to 1 float) */
#define SWE_FORCING_FIELD 2  /* [1|B,1,ny,nx]; batch given by *_batch */

/* Arithmetic of the step kernels (swe_params.arithmetic).
 *   SWE_ARITH_EXACT: every float32 operation of the reference's step, in its
 *     order, IEEE correctly rounded: results equal the reference evaluated
 *     with correctly rounded float32 sqrt/pow, bit for bit.
 *   SWE_ARITH_FAST: the same step within FP32 rounding of the reference
 *     (fused multiply-adds, hardware reciprocal / square root / exp2 / log2
 *     approximations, algebraic identities of the reference's expressions);
 *     about twice the throughput.  After 1000 steps of the 256x256 island
 *     case every field stays within 1.5x the reference's own FP32-vs-FP64
 *     difference of the FP64 reference, with identical wet/dry masks.
 * The mode selects the kernels of swe_spatial_operator_f32, the swe_step_*
 * entry points, the ensemble and the step adjoint (swe_adj_*); the
 * operator-level entry points are always IEEE. */
#define SWE_ARITH_EXACT 0
#define SWE_ARITH_FAST 1

/* SWEConfig (src/config.py:4-28) plus grid spacing and the arithmetic mode.
 * Values are the Python doubles; the library rounds them to float32 where
 * the reference does. */
typedef struct swe_params {
    double gravity, dry_depth, epsilon, cfl, theta, dx, dy;
    double constant_value;                  /* boundary "constant" */
    int32_t bc_left, bc_right, bc_top, bc_bottom;
    int32_t water_slope_reset, positivity_limiter, apply_friction;
    int32_t friction_model;                 /* 0 manning, 1 roughness length */
    int32_t arithmetic;                     /* SWE_ARITH_EXACT or SWE_ARITH_FAST */
    int32_t reserved;                       /* 0 */
} swe_params;

/* Size in 32-bit words of the reduction/status scratch each step uses:
 * [0] max x wave speed bits, [1] max y wave speed bits, [2] status bits,
 * [3] time step (float bits), [4..7] reserved. */
#define SWE_RED_WORDS 8

/*
 * SWE2D.spatial_operator(U, rainfall_rate, infiltration,
 *                        return_wave_speed=True, boundary_level)
 *   src/solver.py:448-531
 * rhs [B,3,ny,nx] receives the tendency; red[0], red[1] receive the bit
 * patterns of the global maxima of the x and y face wave speeds
 * (solver.py:527-530) and red[2] the status bits.  level holds levelB (1 or
 * B) water levels for "water_level"/"absorbing" sides.  red is cleared by
 * the call.
 */
int swe_spatial_operator_f32(const float* U, const float* bed, int B, int bedB, int ny, int nx,
                             const swe_params* p, const float* level, int levelB,
                             const float* rain, int rain_mode, int rain_batch,
                             const float* infil, int infil_mode, int infil_batch, float* rhs,
                             uint32_t* red, void* stream);

/*
 * SWE2D.step(U, model_time, max_dt, infiltration, boundary_level)
 *   src/solver.py:572-663 (friction by src/friction.py:69-131)
 * One adaptive midpoint step: U_out [B,3,ny,nx].  scratch_k is caller-owned
 * device scratch of B*3*ny*nx floats (the stage-1 tendency); red is
 * SWE_RED_WORDS words of device scratch, cleared by the call, in which the
 * step leaves its time step (red[3], float bits) and status (red[2]).
 * max_dt is the float32 value of the reference's max_dt tensor.
 */
int swe_step_f32(const float* U, const float* bed, int bedB, const float* n, int nB, int B,
                 int ny, int nx, const swe_params* p, const float* level, int levelB,
                 float max_dt, const float* infil, int infil_mode, int infil_batch,
                 float* scratch_k, uint32_t* red, float* U_out, void* stream);

/*
 * The two launches of swe_step_f32, enqueued separately (same arguments):
 * stage 1 clears red and writes the stage-1 tendency and wave-speed maxima;
 * stage 2 derives dt and writes U_out; stage 3 is both, i.e. exactly
 * swe_step_f32.  Callers use the split form to time each kernel with stream
 * events.  Same reference lines as swe_step_f32.
 */
int swe_step_stage_f32(int stage, const float* U, const float* bed, int bedB, const float* n,
                       int nB, int B, int ny, int nx, const swe_params* p, const float* level,
                       int levelB, float max_dt, const float* infil, int infil_mode,
                       int infil_batch, float* scratch_k, uint32_t* red, float* U_out,
                       void* stream);

/*
 * A stage of swe_step_stage_f32 with a rainfall source as well: rain is
 * added to the depth tendency of the stage (solver.py:520-525), given like
 * infiltration (SWE_FORCING_*).  The reference evaluates its rainfall
 * forcing at the step's start time for stage 1 and at t + dt/2 for stage 2
 * (SWE2D.step, src/solver.py:609-643), so a caller with rainfall enqueues
 * stage 1, reads dt from red[3], and enqueues stage 2 with the second
 * field.  Same reference lines as swe_step_f32.
 */
int swe_step_stage_forced_f32(int stage, const float* U, const float* bed, int bedB,
                              const float* n, int nB, int B, int ny, int nx, const swe_params* p,
                              const float* level, int levelB, float max_dt, const float* rain,
                              int rain_mode, int rain_batch, const float* infil, int infil_mode,
                              int infil_batch, float* scratch_k, uint32_t* red, float* U_out,
                              void* stream);

/* ---------------------------------------------------------------------
 * Device-driven time loop (SWE2D.forward, src/solver.py:680-779).
 * --------------------------------------------------------------------- */

/* Clock of one forward() call, kept in device memory.  The host fills the
 * first six fields (and zeroes the rest) before the first swe_clock_f32;
 * the device advances it one step at a time, in double precision, exactly
 * as the reference's Python loop does. */
typedef struct swe_clock {
    double duration;   /* t_end of the call (a duration)                      */
    double start;      /* absolute start time                                 */
    double tolerance;  /* max(1e-12, 1e-12 |duration|), solver.py:739          */
    double max_dt_cap; /* > 0: cap on each step's max_dt (solver.py:748-749)   */
    double elapsed;    /* time advanced so far                                 */
    int32_t max_steps; /* RuntimeError bound, solver.py:741, :776-779          */
    int32_t steps;     /* steps taken                                          */
    int32_t active;    /* the next step runs                                   */
    int32_t state;     /* SWE_CLOCK_* below                                    */
    uint32_t dt_status;/* status bits of the failed step (SWE_S_*)             */
    float max_dt;      /* float32 max_dt of the next step                      */
    float level;       /* interpolated boundary level of the next step         */
    float last_dt;     /* dt of the last step taken                            */
} swe_clock;

#define SWE_CLOCK_RUNNING 0
#define SWE_CLOCK_DONE 1      /* remaining time <= tolerance                   */
#define SWE_CLOCK_MAXSTEPS 2  /* max_steps taken before the duration elapsed    */
#define SWE_CLOCK_FAILED 3    /* a step raised (dt_status holds SWE_S_* bits)   */

/*
 * swe_clock_f32: the bookkeeping between two steps of forward().  If the
 * previous step ran: read its dt and status from red, elapsed += dt with
 * the end-of-call clamp (solver.py:766-768), steps += 1, and record the
 * depth of batch 0 at the ngauge cells gauge_cells[2*g], gauge_cells[2*g+1]
 * (row, column) of U into the ring gauges[row*(2+ngauge)+...] as (absolute
 * time, dt, depths...) with row = (steps - 1) % gauge_rows
 * (SWE2D._record_gauges, solver.py:781-801).  Then set up the next step:
 * stop when max_steps steps are taken or the remaining time is within
 * tolerance (solver.py:741-744), else max_dt = remaining (capped), and when nseries
 * > 0 the boundary level at the current time interpolated from the series
 * (SWE2D._interpolate_dynamic_boundary, solver.py:391-415) into *level_out;
 * clear the reduction words of red.  One block; no host synchronisation.
 */
int swe_clock_f32(swe_clock* clock, uint32_t* red, const float* series_t, const float* series_w,
                  int nseries, float* level_out, const float* U, int ny, int nx,
                  const int32_t* gauge_cells, int ngauge, double* gauges, int gauge_rows,
                  void* stream);

/*
 * Clock of a gauge run: n_out output intervals of out_dt seconds, each run
 * exactly like one forward(U, t_end=out_dt, boundary_level=levels[c]) call
 * (the per-chunk model run of the reference's inversion script,
 * Examples/inverse/Monai_Valley/Monai_Velley_BC_inversion_spline_lr002/
 * bc_inversion_train.py:332-411), with the gauges read after the last step
 * of every interval.  base is what the clocked step kernels read; the host
 * fills base.duration = out_dt, base.tolerance, base.max_dt_cap,
 * base.max_steps (per interval), out_dt, n_out and record_cap, and zeroes
 * the rest.
 *
 * Replay mode (replay = 1): the clock re-runs recorded steps
 * [base.steps, replay_end) of an earlier run, each with its recorded dt as
 * max_dt and its interval's level, so the recomputed states are the
 * original ones bit for bit (the CFL dt of the same state is the same
 * float, and min(cfl, dt) = dt).
 */
typedef struct swe_run_clock {
    swe_clock base;
    double out_dt;
    int32_t n_out;
    int32_t chunk;       /* current interval */
    int32_t chunk_steps; /* steps taken in the current interval */
    int32_t record_cap;  /* capacity of step_dt / step_code */
    int32_t replay;      /* 1: replay recorded steps */
    int32_t replay_end;  /* replay: one past the last step to re-run */
} swe_run_clock;

#define SWE_CLOCK_RECORD_FULL 4 /* more steps than record_cap: nothing recorded past it */

/*
 * swe_run_clock_f32: the bookkeeping between two steps of a gauge run.
 * Run mode: after a step, elapsed += dt (with the end-of-call clamp of
 * solver.py:766-768) and the step is recorded as step_dt[s] = dt,
 * step_code[s] = 2*interval + (1 if the step ends its interval); at the end
 * of an interval gauge_out[(b*n_out + c)*ngauge + g] = h + bed at gauge cell
 * (gauge_cells[2g], gauge_cells[2g+1]) of U (the state after the step) for
 * every batch member b, and the next interval starts (elapsed = 0).  Then
 * the next step is set up as swe_clock_f32 does, with the interval's level
 * levels[c*levelB + b] copied into level_out[levelB].  Replay mode: as
 * described at swe_run_clock.  One block; no host synchronisation.
 */
int swe_run_clock_f32(swe_run_clock* clock, uint32_t* red, const float* levels, int levelB,
                      float* level_out, const float* U, const float* bed, int bedB, int B, int ny,
                      int nx, const int32_t* gauge_cells, int ngauge, float* gauge_out,
                      float* step_dt, int32_t* step_code, void* stream);

/*
 * Adjoint of the gauge reads of interval c: lam[b,0,gy,gx] +=
 * g_gauge[(b*n_out + c)*ngauge + g] for every batch member and gauge (the
 * bed term of eta = h + bed is not differentiated).  Gauge cells may
 * repeat.  One block.
 */
int swe_gauge_adjoint_f32(float* lam, int B, int ny, int nx, const int32_t* gauge_cells,
                          int ngauge, const float* g_gauge, int n_out, int c, void* stream);

/*
 * Per-step setup of a device-driven gauge-run backward pass, so a segment of
 * adjoint steps can be captured in one CUDA graph: with s = *cursor,
 * code = step_code[s], c = code >> 1: dt_out[0] = step_dt[s],
 * level_out[b] = levels[c*levelB + b], and if code & 1 (step s ended
 * interval c) the gauge adjoint of swe_gauge_adjoint_f32 is added to lam.
 * A cursor outside [0, nsteps) (the recorded steps) does nothing.  One block.
 */
int swe_gauge_adjoint_prep_f32(const int32_t* cursor, const float* step_dt,
                               const int32_t* step_code, const float* levels, int levelB,
                               float* dt_out, float* level_out, float* lam, int B, int ny, int nx,
                               const int32_t* gauge_cells, int ngauge, const float* g_gauge,
                               int n_out, int nsteps, void* stream);

/*
 * Per-step finish: g_levels[c*levelB + b] += the sum over nparts and blocks
 * of parts[(part*B + b)*blocks + k] (summed over b as well when levelB = 1),
 * c the interval of step *cursor; then *cursor -= 1.  One block.
 */
int swe_gauge_adjoint_post_f32(int32_t* cursor, const int32_t* step_code, const float* parts,
                               int nparts, int B, int blocks, int levelB, float* g_levels,
                               int nsteps, void* stream);

/*
 * One stage (1, 2 or 3 = both) of a step driven by a device clock: like
 * swe_step_stage_f32 but max_dt comes from clock->max_dt and a step whose
 * clock is not active does nothing except copy U to U_out in stage 2.  The
 * reduction words are cleared by swe_clock_f32, not here.  hmax (optional,
 * [B,ny,nx]) receives max(hmax, h_new) (solver.py:765).
 */
int swe_step_clocked_f32(int stage, const float* U, const float* bed, int bedB, const float* n,
                         int nB, int B, int ny, int nx, const swe_params* p, const float* level,
                         int levelB, const swe_clock* clock, const float* infil, int infil_mode,
                         int infil_batch, float* scratch_k, uint32_t* red, float* U_out,
                         float* hmax, void* stream);

/*
 * swe_step_clocked_f32 (stage 2 or 3) that also writes stage 2's tendency
 * k2 = rhs(P) at the predictor P (solver.py:641) into k2_out [B,3,ny,nx],
 * as the step computes it, for an adjoint pass that then need not
 * re-evaluate it.  Steps the clock marks inactive leave k2_out untouched.
 * SWE_EARG with the tiled IEEE kernels (SWE_STEP_KERNEL=tiled).
 */
int swe_step_clocked_k2_f32(int stage, const float* U, const float* bed, int bedB, const float* n,
                            int nB, int B, int ny, int nx, const swe_params* p, const float* level,
                            int levelB, const swe_clock* clock, const float* infil, int infil_mode,
                            int infil_batch, float* scratch_k, uint32_t* red, float* U_out,
                            float* hmax, float* k2_out, void* stream);

/* ---------------------------------------------------------------------
 * Adjoint of the step (the reference's autograd gradient through
 * SWE2D.step, src/solver.py:572-663, with dt detached as in :626).  The
 * arithmetic follows p->arithmetic: SWE_ARITH_EXACT evaluates the adjoint
 * with correctly-rounded quotients and roots, SWE_ARITH_FAST with the
 * hardware approximations of the tolerance-mode step.
 * --------------------------------------------------------------------- */

/*
 * Adjoint of SWE2D.spatial_operator (src/solver.py:448-531) at state S with
 * respect to S and the boundary level: lam_S += (d rhs / d S)^T lam_rhs.
 * scratch_cx holds B*ny*(nx+1)*12 floats, scratch_cy B*(ny+1)*nx*12.
 * level_part receives level_blocks partial sums per batch member
 * ([B][level_blocks]); their sum is the level adjoint of batch member b
 * (summed over b when levelB = 1).  Deterministic (no float atomics).
 */
int swe_adj_spatial_f32(const float* S, const float* bed, int bedB, int B, int ny, int nx,
                        const swe_params* p, const float* level, int levelB,
                        const float* lam_rhs, float* scratch_cx, float* scratch_cy, float* lam_S,
                        float* level_part, int level_blocks, void* stream);

/*
 * swe_adj_spatial_f32 plus the adjoint of the bed (the DEM-correction
 * inversion's gradient, src/solver.py:111-147 under autograd):
 * lam_bed[b,j,i] += d(rhs)/d(bed[b or 0, j, i])^T lam_rhs, per batch member
 * ([B,ny,nx]; the caller sums over b when bedB = 1).  The bed enters through
 * eta = h + z, its limited increments and face values, the Audusse bed,
 * the well-balanced sources and the ghost cells (replicated or periodic
 * copies, forced depth max(level - z, 0)).  Scratch as above but 16 floats
 * per face (B*ny*(nx+1)*16 and B*(ny+1)*nx*16).
 */
int swe_adj_spatial_bed_f32(const float* S, const float* bed, int bedB, int B, int ny, int nx,
                            const swe_params* p, const float* level, int levelB,
                            const float* lam_rhs, float* scratch_cx, float* scratch_cy,
                            float* lam_S, float* level_part, int level_blocks, float* lam_bed,
                            void* stream);

/*
 * Stage 2's spatial adjoint and predictor adjoint together: with
 * P = clean(U, U + dt/2 k1) the step's predictor (solver.py:639) and lam_k2
 * the adjoint of k2 = rhs(P), lam_U += (dP/dU)^T lam_P and
 * lam_k1 = (dP/dk1)^T lam_P (written), where lam_P = (d rhs / d P)^T lam_k2
 * is formed per cell and not stored.  The same result as
 * swe_adj_spatial_f32(P, ..., lam_S = a zeroed lam_P) followed by
 * swe_adj_pointwise_f32(mode 1, U, k1, ..., lam_out = lam_P), in two
 * launches instead of three.  dt_dev, if not null, holds the step's dt in
 * device memory (read in place of dt, for captured graphs).  lam_bed may be
 * null; if not, the bed's adjoint is accumulated as in
 * swe_adj_spatial_bed_f32 (with its 16-float scratch records).  lam_k1 may
 * be the lam_k2 buffer itself (it is written after the last read of lam_k2).
 */
int swe_adj_stage2_f32(const float* P, const float* U, const float* k1, const float* bed, int bedB,
                       int B, int ny, int nx, const swe_params* p, const float* level, int levelB,
                       const float* lam_k2, float* scratch_cx, float* scratch_cy, float dt,
                       const float* dt_dev, float* lam_U, float* lam_k1, float* level_part,
                       int level_blocks, float* lam_bed, void* stream);

/*
 * Pointwise parts of the step adjoint, for step input U, tendency k and
 * time step dt:
 *   mode 0: corrector and friction (solver.py:646-661, friction.py:12-131):
 *           lam_out = adjoint of the step output; lam_U += ..., lam_k = adjoint
 *           of k2, lam_n += adjoint of the roughness field [nB,1,ny,nx];
 *   mode 1: predictor (solver.py:639): lam_out = adjoint of P; lam_U += ...,
 *           lam_k = adjoint of k1;
 *   mode 2: forward predictor P_out = clean(U, U + dt/2 k) (for recompute);
 *   mode 3: mode 0 with lam_U written (=) instead of accumulated, for a
 *           lam_U that starts the step's accumulation (no zeroing pass).
 */
int swe_adj_pointwise_f32(int mode, const float* U, const float* k, const float* n, int nB, int B,
                          int ny, int nx, const swe_params* p, float dt, const float* lam_out,
                          float* lam_U, float* lam_k, float* lam_n, float* P_out, void* stream);

/* swe_adj_pointwise_f32 with the time step read from device memory
 * (*dt_dev), for launches captured in a CUDA graph whose step varies. */
int swe_adj_pointwise_dev_f32(int mode, const float* U, const float* k, const float* n, int nB,
                              int B, int ny, int nx, const swe_params* p, const float* dt_dev,
                              const float* lam_out, float* lam_U, float* lam_k, float* lam_n,
                              float* P_out, void* stream);

/* ---------------------------------------------------------------------
 * Ensembles: many independent scenarios in one persistent launch.
 * (No counterpart in the reference, whose batch dimension requires equal
 * grid sizes and shares one time step, src/solver.py:367-376, :527-530.)
 * --------------------------------------------------------------------- */

/* One scenario: its own grid, bed, roughness, configuration, boundary level
 * (constant or a series) and step count; every time step is its own CFL
 * step (capped by max_dt).  Device pointers; the state starts in U_a and
 * after `steps` steps is in U_a (even steps) or U_b (odd).
 *
 * Interval mode (n_out > 0): the member runs n_out output intervals of
 * out_dt seconds exactly as swe_run_clock_f32 does (each interval like one
 * forward(t_end=out_dt) call with level out_levels[c]; max_dt, if > 0, caps
 * each step), writes eta = h + bed at its gauge cells after every interval
 * into gauge_out[c*ngauge + g], and stops after the last interval; `steps`
 * is then a cap (reaching it first fails the member with SWE_S_STEP_LIMIT);
 * nseries and level are ignored. */
typedef struct swe_ensemble_member {
    const float* bed;       /* [ny,nx] */
    const float* n;         /* [ny,nx] Manning n or roughness length */
    float* U_a;             /* [3,ny,nx] state (initial state on entry) */
    float* U_b;             /* [3,ny,nx] second state buffer */
    float* k1;              /* [3,ny,nx] scratch */
    float* hmax;            /* [ny,nx] running max depth, or NULL */
    const float* series_t;  /* boundary series times (float32), or NULL */
    const float* series_w;  /* boundary series levels */
    int32_t nseries;        /* 0: constant `level` */
    int32_t ny, nx;
    int32_t steps;          /* steps to run */
    int32_t rows;           /* output rows per sweep tile (autotuned) */
    float level;            /* constant boundary level when nseries == 0 */
    double start_time;      /* absolute time of the initial state */
    double max_dt;          /* cap on each step (float32-rounded) */
    swe_params params;      /* all members share apply_friction / friction_model */
    double out_dt;          /* interval mode: seconds per output interval */
    int32_t n_out;          /* interval mode: intervals (0: step-count mode) */
    int32_t ngauge;         /* gauge cells */
    const float* out_levels;     /* [n_out] boundary level of each interval */
    const int32_t* gauge_cells;  /* [2*ngauge] (row, column) */
    float* gauge_out;            /* [n_out*ngauge] eta after each interval */
} swe_ensemble_member;

#define SWE_ENSEMBLE_MAX_GAUGES 64

typedef struct swe_ensemble_result {
    int32_t steps;     /* steps completed */
    int32_t finished;  /* 1 done, 2 failed (status holds SWE_S_* bits) */
    uint32_t status;
    float dt_last;
    double time;       /* simulated time advanced */
} swe_ensemble_result;

/* Device workspace bytes for `count` members (count <= 1024), -1 if invalid. */
long long swe_ensemble_workspace_bytes(int count);

/* Copies the members' description into `workspace` (device) and resets the
 * ensemble's control state.  Setup only: synchronous host-to-device copies. */
int swe_ensemble_prepare_f32(const swe_ensemble_member* members, int count, void* workspace,
                             void* stream);

/* Resets the control state (step counts, times, levels, reductions) so the
 * ensemble can run again from its state buffers.  One small kernel. */
int swe_ensemble_reset_f32(void* workspace, int count, void* stream);

/* Runs every member for its step count in one persistent launch of `blocks`
 * blocks of 128 threads (friction: 0 off, 1 Manning, 2 roughness length;
 * arithmetic: SWE_ARITH_*; both as in the members' params).  Each member's
 * stages are claimed tile by tile from per-member counters; no block waits
 * for a particular item.  Idle polling backs off and is bounded: if no
 * member completes a phase for stall_ns nanoseconds (0: the default, 2 s)
 * the blocks stop and swe_ensemble_results_f32 reports error bit 1.
 * Capturable in a CUDA graph. */
int swe_ensemble_run_f32(void* workspace, int count, int friction, int arithmetic, int blocks,
                         long long stall_ns, void* stream);

/* Per-member results into out[count] (device) and the launch's error word. */
int swe_ensemble_results_f32(const void* workspace, int count, swe_ensemble_result* out,
                             uint32_t* error, void* stream);

/* Loads every step/ensemble kernel's module now (CUDA loads kernels lazily
 * on first launch); call once before capturing launches in a CUDA graph. */
int swe_load_kernels(void);

/* Output rows per tile of the single-grid sweep kernels (process-wide
 * tuning knob, default 64; set it between launches, not during them). */
int swe_tune_sweep_rows(int rows);

/* The current value of that knob (CUDA graphs keep the value they were
 * captured with). */
int swe_sweep_rows(void);

/*
 * swe_step_noalloc_f32 -- one step like swe_step_f32, for callers that must
 * not allocate device memory.  No counterpart in the reference: it exists
 * for hosts whose device memory belongs to another allocator (a framework's
 * caching allocator or memory pool) or that forbid allocation after
 * start-up (a real-time control loop), and so cannot hand the step the
 * scratch_k / red buffers that swe_step_f32 takes.
 *
 * The scratch lives in a static device array inside the library, sized for
 * B*ny*nx <= SWE_NOALLOC_MAX_CELLS cells (12 MiB plus 256 bytes); every GPU
 * that loads the library holds that array until the process exits.  Larger
 * grids are rejected with SWE_ETOOLARGE before anything is enqueued.
 * The call allocates nothing: it issues one memset and the two step kernels
 * on `stream`, and copies the step's status word and time step (float
 * bits) into status_dt[0..1] (device memory, provided by the caller).
 * The first call on a device looks up the array's device address with that
 * device current (once per device, cached); make that first call before
 * any stream capture.  All calls share the one array and it keeps the last
 * call's contents (the call clears the words that must start at zero), so
 * calls that overlap on the GPU -- on different streams, or from different
 * host threads without ordering -- race and give wrong results.
 */
#define SWE_ETOOLARGE 3 /* grid larger than the static scratch of the no-alloc step */
#define SWE_NOALLOC_MAX_CELLS (1 << 20)

int swe_step_noalloc_f32(const float* U, const float* bed, int bedB, const float* n, int nB,
                         int B, int ny, int nx, const swe_params* p, const float* level,
                         int levelB, float max_dt, const float* infil, int infil_mode,
                         int infil_batch, float* U_out, uint32_t* status_dt, void* stream);

/* ---------------------------------------------------------------------
 * Operator-level entry points (the reference's numerical operators).
 * --------------------------------------------------------------------- */

/*
 * add_ghost_cells(U, bed, ng, boundary_*, constant_value, constant_level)
 *   src/boundary.py:150-413
 * Up [B,3,ny+2ng,nx+2ng] and zp [bedB,1,ny+2ng,nx+2ng], including the
 * corner cells as the reference's left/right/top/bottom overwrites leave
 * them.  level and constant_value hold levelB / cvalB (1 or B) values.
 */
int swe_ghost_cells_f32(const float* U, const float* bed, int B, int bedB, int ny, int nx, int ng,
                        const swe_params* p, const float* level, int levelB,
                        const float* constant_value, int cvalB, float* Up, float* zp,
                        void* stream);

/*
 * bflood_cn_reconstruction(U, bed, dim, gravity, epsilon, dry_depth, theta,
 *                          water_slope_reset)   src/reconstruction.py:18-108
 * Up [B,3,H,W], zp [zB,1,H,W]; dim = -1 (x) or -2 (y), with torch.roll
 * wrap-around at the array ends.  UL, UR [B,3,H,W]; sL, sR [B,1,H,W].
 */
int swe_reconstruction_f32(const float* Up, const float* zp, int B, int zB, int H, int W, int dim,
                           const swe_params* p, float* UL, float* UR, float* sL, float* sR,
                           void* stream);

/*
 * bflood_hllc_flux(UL, UR, normal, gravity, epsilon, dry_depth)
 *   src/riemann.py:41-105
 * UL, UR [B,3,H,W] -> flux [B,3,H,W], speed [B,1,H,W]; normal_y = 0 for
 * "x", 1 for "y".
 */
int swe_hll_flux_f32(const float* UL, const float* UR, int B, int H, int W, int normal_y,
                     const swe_params* p, float* flux, float* speed, void* stream);

/* primitive(U, gravity, epsilon, dry_depth)   src/riemann.py:20-38
 * U [B,3,H,W] -> h, u, v, c [B,1,H,W]. */
int swe_primitive_f32(const float* U, int B, int H, int W, const swe_params* p, float* h,
                      float* u, float* v, float* c, void* stream);

/* limited_increment(q, dim, theta)   src/numerics.py:16-27
 * q is `outer` contiguous [H,W] planes; dim = -1 or -2 (roll wrap-around). */
int swe_limited_increment_f32(const float* q, int outer, int H, int W, int dim, double theta,
                              float* out, void* stream);

/* minmod3(a, b, c)   src/numerics.py:4-13, elementwise over n values. */
int swe_minmod3_f32(const float* a, const float* b, const float* c, long long n, float* out,
                    void* stream);

/* SWE2D._clean_and_limit(old, candidate)   src/solver.py:547-570 */
int swe_clean_and_limit_f32(const float* old, const float* cand, int B, int ny, int nx,
                            const swe_params* p, float* out, void* stream);

/*
 * apply_manning_friction (model 0)      src/friction.py:102-131
 * apply_roughness_length_friction (1)   src/friction.py:69-99
 * U [B,3,ny,nx], n (Manning n or roughness length) [nB,1,ny,nx]; dt is
 * the float32 time step; p->dry_depth and p->epsilon are the functions'
 * dry_depth / epsilon arguments.
 */
int swe_friction_f32(const float* U, const float* n, int nB, int B, int ny, int nx, float dt,
                     int model, const swe_params* p, float* out, void* stream);

/*
 * Device self-test of the step's division, square root and friction power
 * (no counterpart in the reference; it checks that the step's arithmetic is
 * the IEEE correctly-rounded arithmetic of the reference's float32 tensors).
 * which = 0: reciprocal, exhaustive over |b| in [2^-100, 2^100);
 * which = 1: division on n random operand pairs (seed);
 * which = 2: division on n operand pairs built next to rounding midpoints;
 * which = 3: square root, exhaustive over [2^-100, 2^100);
 * which = 4: x ** t (t = the float with the bit pattern seed & 0xffffffff)
 *            against the double pow rounded to float, every x in
 *            [2^-40, 2^14);
 * which = 5: division with numerators below 2^-62 (subnormals included) on
 *            n draws of six operand pairs.
 * count (device, 1 x u64) receives the number of mismatches against CUDA's
 * rcp.rn / div.rn / sqrt.rn / pow, first (device, 2 x u32) the first bad
 * input.
 */
int swe_selftest_arith_f32(int which, long long n, unsigned long long seed,
                           unsigned long long* count, uint32_t* first, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* SWE_B200_H */
