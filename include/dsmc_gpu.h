/*
 * dsmc_gpu.h — C ABI of the B200 DSMC particle step.
 *
 * Drop-in boundary for the DSMC member functions that the reference's driver
 * (src/meshImportTest.cpp:171-234), dynamicDSMC and ProcessGSIS call on
 * ProcessDSMC (src/ProcessDSMC.h:441-492). The host keeps the mesh import and
 * the macroscopic GSIS / NS-G13 step; one handle holds one case (mesh,
 * particles, per-cell collision and sampling state) resident on one GPU.
 *
 * Conventions
 *   - Every entry point returns 0 on success or a negative DSMC_E_* code; no
 *     C++ exception crosses this boundary. dsmc_last_error() gives the text.
 *   - Host buffers are owned by the caller and only accessed during the call.
 *   - Array layouts are the reference's: per-cell macro fields are
 *     [cell][18] doubles in MacroIndex order (src/ProcessDSMC.h:28-49), the
 *     mesh arrays are DsmcCell[] / DsmcEdge[] / localPointXY[3*npoint] /
 *     faceSplitTag[nface] (src/meshImport.h:168-189), case constants are a
 *     meshMessage image (src/meshImport.h:192-208).
 *   - One domain: local cell id == global cell id, one compute "rank".
 *   - A handle is used by one host thread at a time (or externally
 *     serialised); its work runs on one CUDA stream it owns.
 */
#ifndef DSMC_GPU_H
#define DSMC_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
#define DSMC_OK              0
#define DSMC_E_INVALID      -1   /* bad argument / inconsistent mesh        */
#define DSMC_E_CUDA         -2   /* CUDA runtime error                      */
#define DSMC_E_NOMEM        -3   /* device allocation failed                */
#define DSMC_E_CAPACITY     -4   /* particle store overflow                 */
#define DSMC_E_DEVICE_FAULT -5   /* kernel-reported error (see counters)    */
#define DSMC_E_STATE        -6   /* call out of order                       */

/* ---- mesh records: byte layout of the reference's structs --------------- */
/* DsmcCell, src/meshImport.h:168-178 (120 bytes) */
typedef struct DsmcCellRec {
    int32_t num;
    int32_t fluentCellType;
    int32_t cell2face[6];
    int32_t cell2cell[6];
    int32_t cell2face_sgn[6];
    double  area;             /* cell VOLUME (src/meshImport.cpp:719) */
    int32_t no;
    double  cellXY[3];
} DsmcCellRec;

/* DsmcEdge, src/meshImport.h:180-189 (88 bytes); faceMap[4..5] = c0, c1 */
typedef struct DsmcEdgeRec {
    int32_t faceTag;
    int32_t faceType;
    double  length;           /* face area */
    int32_t faceMap[6];
    double  edgeNormal[3];    /* unit, from c0 to c1 */
    double  edgeCenter[3];
} DsmcEdgeRec;

/* meshMessage, src/meshImport.h:192-208 (344 bytes) */
typedef struct DsmcMeshMessage {
    int32_t Ncell, Nface, Npoint, Nk, bcnumber, Nghost;
    double Area;
    double Ma, Kn, cfl;
    double gamma, dr, dv, zr, zv, omega;
    int32_t var, qn;
    double f_tra, f_rot;
    double delta_rp, delta_sm, omeag0, omeag1;
    double cfl_ns, pr, cp, cv;
    double kB, p_mass, p_mass_r, T_ref, n_ref, miu_ref, Twall_ref, p_ref, d_ref;
    double alpha, v_rms, eta, P_relax, dt_ref;
    double T_in, v_in;
    int32_t eNface, iNface;
    double Neff;
    double dtime;
} DsmcMeshMessage;

typedef struct DsmcMeshDesc {
    int32_t ncell;
    int32_t nface;
    int32_t npoint;
    const DsmcCellRec* cells;          /* [ncell] */
    const DsmcEdgeRec* edges;          /* [nface] */
    const double* localPointXY;        /* [3*npoint] */
    const unsigned char* faceSplitTag; /* [nface], FACE_SPLIT_02/13/255 */
} DsmcMeshDesc;

/* DSMC role of a Fluent zone tag (BoundaryRole, src/BoundaryCondition.h:10-24;
 * SPECULAR is this library's addition: mirror reflection, no reference
 * counterpart, where the reference leaves the tag unmapped). */
enum DsmcRole {
    DSMC_ROLE_NONE = 0,
    DSMC_ROLE_INTERFACE = 1,
    DSMC_ROLE_INLET = 2,
    DSMC_ROLE_OUTLET = 3,
    DSMC_ROLE_WALL = 4,
    DSMC_ROLE_SPECULAR = 5
};

enum DsmcPrecision {
    DSMC_PRECISION_FP64 = 0,   /* all-FP64 state and arithmetic (reference) */
    DSMC_PRECISION_MIXED = 1   /* FP32 state/trace/collide, FP64 fallback
                                  and FP64 accumulators */
};

#define DSMC_MAX_ZONES 16

/* Controls that are compile-time constants or hard-coded values in the
 * reference (src/meshImport.h:45-58, src/ProcessDSMC.cpp:2330-2331,
 * src/BoundaryCondition.h:79-117). dsmc_default_params() fills the
 * reference's values. */
typedef struct DsmcCaseParams {
    int32_t precision;            /* DsmcPrecision */
    int32_t nss;                  /* NSS: steady sampling starts after it   */
    int32_t nscheme;              /* NSCHEME: exponential-average window    */
    int32_t nevery;               /* Nevery                                 */
    int32_t nrepeat;              /* Nrepeat (NGSIS = nevery*nrepeat)       */
    int32_t wall_stats;           /* EnableBoundaryStressHeatStatistic      */
    double  inflow_dir[2];        /* drift direction (x,y); reference 30 deg */
    int32_t nzones;
    int32_t zone_tag[DSMC_MAX_ZONES];
    int32_t zone_role[DSMC_MAX_ZONES];   /* DsmcRole */
    int32_t zone_inject[DSMC_MAX_ZONES]; /* inlet zones that emit particles */
    int64_t capacity;             /* particle store size; 0 = automatic      */
    uint64_t seed;                /* Philox key                              */
    int32_t max_crossings;        /* per particle per step; lost beyond it   */
    int32_t keep_step_moments;    /* keep last step's raw moments on device  */
} DsmcCaseParams;

/* Stage flags of dsmc_step, in the reference's step order
 * (src/meshImportTest.cpp:207-234). */
#define DSMC_STAGE_INJECT   0x1u   /* preprocesseffquad */
#define DSMC_STAGE_MOVE     0x2u   /* advection         */
#define DSMC_STAGE_SORT     0x4u   /* cache2chain       */
#define DSMC_STAGE_COLLIDE  0x8u   /* collisionDSMC     */
#define DSMC_STAGE_SAMPLE   0x10u  /* statistic_macro   */
#define DSMC_STAGE_ALL      0x1Fu

/* dsmc_download_macro targets (ProcessDSMC::local/record/final_record) */
#define DSMC_MACRO_LOCAL        0
#define DSMC_MACRO_RECORD       1
#define DSMC_MACRO_FINAL_RECORD 2
#define DSMC_MACRO_WIDTH        18

/* cumulative device counters, dsmc_get_counters() */
typedef struct DsmcCounters {
    uint64_t steps;
    uint64_t injected;          /* particles emitted by inlet patches        */
    uint64_t removed;           /* left through an inlet / outlet face       */
    uint64_t dropped;           /* no exit face found (reference "Dropped")  */
    uint64_t lost;              /* crossing cap hit or bad neighbour         */
    uint64_t wall_hits;
    uint64_t crossings;         /* face crossings of all kinds               */
    uint64_t candidate_pairs;   /* NTC pairs (tol_collision_pairs)           */
    uint64_t collisions;        /* accepted pairs (tol_collision_times)      */
    uint64_t fp64_fallbacks;    /* mixed path: crossing steps redone in FP64 */
    uint64_t overflow;          /* particles not stored: capacity exceeded   */
    uint64_t big_cells;         /* cells sorted with more than 512 particles */
} DsmcCounters;

typedef struct DsmcHandle DsmcHandle;

/* Fill *p with the reference's compile-time values. Replaces the constants
 * at src/meshImport.h:45-58 and the boundary table of
 * src/BoundaryCondition.h:79-117. */
void dsmc_default_params(DsmcCaseParams* p);

/* Build a case: copies the mesh, builds the per-cell triangle cache
 * (rebuildFaceTraversalCache, src/ProcessDSMCGeometry.cpp:145-214), the
 * face-cross cache (src/ProcessDSMCGeometry.cpp:114-136), wall normals
 * (processFacesQuadNormals, src/ProcessDSMC.cpp:1054-1127) and inlet emit
 * patches (rebuildBoundaryEmitCache, src/ProcessDSMC.cpp:583-768), and
 * allocates all device state. Replaces ProcessDSMC::ProcessDSMC
 * (src/ProcessDSMC.cpp:271-288) plus Collision_constant_initial
 * (src/MeshparticalInitial.cpp:798-810). device < 0 uses the current one. */
int dsmc_create(const DsmcMeshDesc* mesh, const DsmcMeshMessage* mess,
                const DsmcCaseParams* params, int device, DsmcHandle** out);

void dsmc_destroy(DsmcHandle* h);

/* Text of the last error on this handle (or of the last failed create when
 * h is NULL). */
const char* dsmc_last_error(const DsmcHandle* h);

/* Replace all particles (the buckets cell_particles_curr,
 * src/MeshparticalInitial.h:229) with n particles given as SoA host arrays.
 * cell[] are local cell ids. Particles are binned and canonically ordered on
 * the device. */
int dsmc_upload_particles(DsmcHandle* h, int64_t n,
                          const double* px, const double* py, const double* pz,
                          const double* vx, const double* vy, const double* vz,
                          const double* ir, const int32_t* cell);

/* Replace all particles by the reference's initial fill, made on the device
 * (MeshparticalInitial's constructor fill: Np_tri_inititial / meshfillpar /
 * velocityLocationGenerate, src/MeshparticalInitial.cpp:413-418, 481-721,
 * with the per-cell counts of setParticleMessage, src/meshImport.cpp:
 * 1399-1421). Cell c gets Np = floor(Ns) or floor(Ns) + 1 particles (the
 * latter with probability frac(Ns)), Ns = V_c * ppc_mean * ncell / V_total.
 * The cell is split into placement tetrahedra as buildCellInitTets does
 * (a tetrahedral cell is one; a pyramid two, base triangles with the apex;
 * other cells the centre with each face triangle); tetrahedron t gets
 * Iround(Np V_t / V_cell) particles, adjusted by +-1 on randomly chosen
 * tetrahedra to sum to Np (adjust_particles, clamped at zero). A particle
 * is the point a V0 + b V1 + c V2 + d V3 of its tetrahedron with (a, b, c,
 * d) four uniforms divided by their sum (randomBarycentric4; not uniform in
 * the tetrahedron, denser towards its centroid, as in the reference), a unit
 * Maxwellian velocity at rest (Box-Muller: sqrt(-2 ln r) sin th,
 * sqrt(-2 ln r) cos th, sqrt(-2 ln r2) sin th2) and Ir = -ln(r3) / 2.
 * seed keys the fill's random streams (Philox). */
int dsmc_fill_initial(DsmcHandle* h, double ppc_mean, uint64_t seed);

/* dsmc_fill_initial's counts and placement with the case's freestream
 * instead of the unit Maxwellian at rest: drift Ma sqrt(gamma/2) v_in / v_rms
 * along the inflow direction, thermal spread sqrt(T/2) per component and
 * Ir = -ln(r3) T / 2, T = T_in / T_ref (computeBoundaryGasState,
 * src/ProcessDSMC.cpp:2318-2367). This is the state the reference's coupled
 * start-up reaches when its first GSIS update shifts the fill to a uniform
 * freestream (dsmc_molecular_velocity_change does the same on the device).
 * The freestream number density corresponds to ppc_mean equal to the
 * particles per cell the case's Neff was set for (meshMessage). */
int dsmc_fill_freestream(DsmcHandle* h, double ppc_mean, uint64_t seed);

/* Outcome of a GSIS particle update. */
typedef struct DsmcGsisReport {
    int32_t nan_cell;        /* first cell with a NaN NS density or velocity (the
                                update stops before it), -1 when there is none */
    int32_t cells_updated;   /* cells brought to their NS state */
    int32_t cells_skipped;   /* cells the acceptance gate left alone */
    int32_t pad;
    int64_t added;           /* particles copied or sampled */
    int64_t removed;         /* particles deleted */
    int64_t particles;       /* particles after the update */
} DsmcGsisReport;

/* The GSIS particle update between two steps, on the device
 * (ProcessGSIS::molecular_velocity_change with replication, deletion,
 * MaxwellianSample and randomlocation, src/ProcessGSIS.cpp:2239-2530).
 * nsresult [ncell][6]: the NS solution per cell, density / n_ref, velocity
 * (3), T and Tr in the particle state's normalisation. accepted [ncell] or
 * NULL: when given (the acceptance gate is on) cells with accepted[c] == 0
 * are left untouched. Cells are taken in order and the update stops at the
 * first gated-in cell whose density or velocity is NaN (report->nan_cell).
 * Each updated cell is brought to Iround(density V_c n_ref / Neff)
 * particles, by copying particles chosen uniformly from the growing bucket
 * to random points of the cell (sampling a Maxwellian at the NS state when
 * the cell is empty, unless T < 0) or by deleting uniformly chosen
 * particles (the last one fills the hole); a deletion of more particles
 * than the cell holds (negative density) is refused, as in the reference.
 * Then v -> k v + b and Ir -> kr Ir with k = sqrt(T_ns / T), b = u_ns - k u,
 * kr = Tr_ns / Tr from the cell's moments (T = 2/(3N) (sum v^2 - N u^2),
 * Tr = 4 / dr / N sum Ir), when T, T_ns and Tr are positive. Random
 * choices come from Philox streams keyed by the case's seed, the cell and
 * the update's sequence number on this handle. Grows the particle store
 * when automatic (DSMC_E_CAPACITY with a fixed capacity); a density that
 * gives a count outside [0, 2^30) leaves the particles untouched and
 * returns DSMC_E_INVALID. report may be NULL. */
int dsmc_molecular_velocity_change(DsmcHandle* h, const double* nsresult, const char* accepted,
                                   DsmcGsisReport* report);

/* Particle count (sum of bucket sizes). */
int dsmc_particle_count(DsmcHandle* h, int64_t* n);

/* Copy all particles back (cell-major, within a cell by particle id). Any
 * pointer may be NULL to skip that array. pid[] are the device particle ids. */
int dsmc_download_particles(DsmcHandle* h, int64_t n,
                            double* px, double* py, double* pz,
                            double* vx, double* vy, double* vz,
                            double* ir, int32_t* cell, uint32_t* pid);

/* One DSMC step, stages selected by DSMC_STAGE_* flags, in reference order.
 * DSMC_STAGE_ALL is the fused production path (one CUDA graph). */
int dsmc_step(DsmcHandle* h, int32_t istep, uint32_t stages);

/* Stage entry points with the reference's member names and arguments
 * (src/ProcessDSMC.h:459-488). Calling the five in order equals
 * dsmc_step(h, istep, DSMC_STAGE_ALL). */
int dsmc_preprocesseffquad(DsmcHandle* h, int32_t istep); /* ProcessDSMC.cpp:2556 */
int dsmc_advection(DsmcHandle* h, int32_t istep);         /* ProcessDSMC.cpp:1946 */
int dsmc_cache2chain(DsmcHandle* h);                      /* ProcessDSMC.cpp:2030 */
int dsmc_collisionDSMC(DsmcHandle* h);                    /* ProcessDSMC.cpp:2621 */
int dsmc_statistic_macro(DsmcHandle* h, int32_t istep);   /* ProcessDSMC.cpp:2757 */
int dsmc_statistic_macroPre(DsmcHandle* h);               /* ProcessDSMC.cpp:3312 */

/* Per-cell macro fields [ncell][18] (local / record / final_record). */
int dsmc_download_macro(DsmcHandle* h, int32_t which, double* out);

/* Per-cell state read by ProcessGSIS::DSMC2NS (src/ProcessGSIS.cpp:1569-1656).
 * Any pointer may be NULL. ppc = particles per cell. */
int dsmc_download_counts(DsmcHandle* h, int32_t* ppc, double* window_samples,
                         char* window_valid, unsigned char* sparse_state,
                         double* stepinter_rho, double* steady_rho);

/* Raw per-cell moment sums [ncell][18] of the last sampled step (requires
 * params.keep_step_moments) in the order
 * N, Σv(3), Σv², Σvv(xx,xy,yy,yz,zz,zx), Σv v²(3), ΣIr, Σv Ir(3). */
int dsmc_download_step_moments(DsmcHandle* h, double* out);

/* Wall surface tallies [nface][6]: hits, Δmomentum(3), ΔE_tr, ΔE_rot
 * (recordBoundaryStressHeat, src/ProcessDSMC.cpp:1659-1689); zero rows for
 * non-wall faces. */
int dsmc_download_wall(DsmcHandle* h, double* tally);

/* Per-cell collision state: crmax, remainderincoll (src/MeshparticalInitial.h:
 * 233-235) and per-cell inflow remainder remainderinpre. Any may be NULL. */
int dsmc_download_cell_state(DsmcHandle* h, double* crmax, double* rem_coll, double* rem_inj);
int dsmc_upload_cell_state(DsmcHandle* h, const double* crmax, const double* rem_coll, const double* rem_inj);

/* Per-cell sparse-sample states [ncell] written back by the host's GSIS
 * exchange: ProcessGSIS::DSMC2NS marks a cell accumulating (1) when its
 * samples are too few or its cell Knudsen number is rejected, and released
 * (2) when an accumulating cell's fields become reliable
 * (src/ProcessGSIS.cpp:1660-1674), in the ProcessDSMC object the step then
 * reads. Values outside 0..2 are refused and nothing is written. */
int dsmc_upload_sparse_state(DsmcHandle* h, const unsigned char* sparse_state);

int dsmc_get_counters(DsmcHandle* h, DsmcCounters* out);

/* Tracing check entry (the move kernel's trace on caller-given particles,
 * no state change): each particle i starts in cell[i] at (p*, v*) with
 * dt[i] to fly, exactly as ParticleTransportOps::traceParticleDtleft
 * (src/ProcessDSMC.cpp:149-221) with a fresh crossing state. With
 * stop_at_wall != 0 a particle stops at its first wall hit instead of being
 * re-emitted. Outputs (any may be NULL): final cell (-1 removed/dropped),
 * ifout (0 stayed, 1 crossed, -1 removed/dropped), first non-interface face
 * and its triangle tag (-1/0 if none), number of crossings, final position,
 * velocity and remaining dt. Runs at the handle's precision. */
int dsmc_trace(DsmcHandle* h, int64_t n,
               const double* px, const double* py, const double* pz,
               const double* vx, const double* vy, const double* vz,
               const double* dt, const int32_t* cell, int32_t stop_at_wall,
               int32_t* out_cell, int32_t* out_ifout, int32_t* out_face,
               int32_t* out_tri, int32_t* out_ncross,
               double* out_px, double* out_py, double* out_pz,
               double* out_vx, double* out_vy, double* out_vz, double* out_dt);

/* Tracing check for callers that cannot allocate device memory at the
 * call site: a solver that reserved the whole device for its own memory
 * pool, or a coupling loop that forbids allocation after start-up so that
 * its memory footprint stays fixed. Same arguments and results as
 * dsmc_trace, but the host arrays are staged in one static device array of
 * the library instead of in buffers allocated per call: the call makes no
 * device allocation (no cudaMalloc, cudaFree or allocating library routine);
 * only its error paths format a message on the host. Limits and caveats:
 *   - n <= DSMC_NOALLOC_MAX_TRACE particles per call (larger n is rejected
 *     with DSMC_E_INVALID); the array takes 7.74 MB (7,737,344 bytes) on
 *     every GPU that loads the library, until the process exits.
 *   - The first call on a device looks up the array's device address (with
 *     that device current); make that first call before any stream capture.
 *   - The call copies from and to the caller's host arrays on the handle's
 *     stream and synchronises that stream before it returns.
 *   - All calls on a device share the array: calls whose work overlaps on the
 *     GPU (other streams, other host threads) race; serialise them.
 * No counterpart in the reference: it is an addition of this library. */
#define DSMC_NOALLOC_MAX_TRACE 32768
int dsmc_trace_noalloc(DsmcHandle* h, int64_t n,
                       const double* px, const double* py, const double* pz,
                       const double* vx, const double* vy, const double* vz,
                       const double* dt, const int32_t* cell, int32_t stop_at_wall,
                       int32_t* out_cell, int32_t* out_ifout, int32_t* out_face,
                       int32_t* out_tri, int32_t* out_ncross,
                       double* out_px, double* out_py, double* out_pz,
                       double* out_vx, double* out_vy, double* out_vz, double* out_dt);

/* Stage timing: with on != 0, dsmc_step runs its kernels without a CUDA
 * graph and records CUDA events between the stages; dsmc_stage_ms then
 * returns the device time of [inject, move, sort, collide, sample] (ms5[5])
 * summed over the timed steps since the last reset (reset != 0 clears the
 * sums after reading). Off (the default) replays one captured graph per
 * step. */
int dsmc_set_timing(DsmcHandle* h, int32_t on);
int dsmc_stage_ms(DsmcHandle* h, double* ms5, int64_t* nsteps, int32_t reset);

/* The CUDA stream the handle's work runs on (a cudaStream_t). */
void* dsmc_stream(DsmcHandle* h);

/* Synchronise the handle's stream and report kernel-side errors. */
int dsmc_sync(DsmcHandle* h);

/* ---------------------------------------------------------------------------
 * Launch shapes and the autotuner. No reference counterpart: the reference
 * runs on CPU cores. Every kernel loops over its work and draws from
 * counter-based random streams, so the shape changes the speed of a step,
 * never its result.
 * ------------------------------------------------------------------------- */
typedef struct DsmcLaunchShape {
    int32_t move_threads;          /* threads per block of the move kernel: 128 or 256 */
    int32_t move_blocks_per_sm;    /* move grid = SMs x this, 1..32 (particles per thread follow) */
    int32_t sort_blocks_per_sm;    /* rank / scatter / gather grids = SMs x this, 1..32 */
    int32_t collide_blocks_per_sm; /* cap on the collision grid per SM, 1..32 (at most the resident blocks; default 32) */
    int32_t stay_per_thread;       /* particles per thread of the move's stay pass: 1, 2 or 4 (default 4) */
} DsmcLaunchShape;

int dsmc_get_launch_shape(DsmcHandle* h, DsmcLaunchShape* out);
/* Takes effect for steps enqueued after the call (captured graphs are rebuilt). */
int dsmc_set_launch_shape(DsmcHandle* h, const DsmcLaunchShape* shape);

/* Runs full steps first_istep, first_istep+1, ... of the case, timing each
 * stage, and keeps per stage the fastest of a few shapes (move: block size
 * x blocks per SM, particles per thread of the stay pass; sort: blocks per
 * SM; collide keeps its cap). The steps
 * are ordinary steps of the case (about 15 x trial_steps of them);
 * *next_istep receives the next step to run, *chosen the shape kept. */
int dsmc_autotune(DsmcHandle* h, int32_t first_istep, int32_t trial_steps, int32_t* next_istep,
                  DsmcLaunchShape* chosen);

/* ---------------------------------------------------------------------------
 * Batched steps: many independent cases (handles on one device, each with
 * its own mesh, constants, particles and step counter) advanced together,
 * each step of all of them replayed as one CUDA graph whose branches run
 * concurrently. No reference counterpart: the reference runs one case per
 * MPI job.
 * ------------------------------------------------------------------------- */
typedef struct DsmcBatch DsmcBatch;

/* The cases must be distinct handles on one device. The batch does not own
 * them; destroy the batch before any of its cases. */
int dsmc_batch_create(DsmcHandle* const* cases, int32_t n, DsmcBatch** out);
void dsmc_batch_destroy(DsmcBatch* b);
const char* dsmc_batch_last_error(const DsmcBatch* b);

/* Advance every case by nsteps full steps; each case's steps continue its
 * own count (the step after its last dsmc_step / stage call / batch step).
 * Equal, bit for bit, to stepping each case on its own. Asynchronous: work
 * queued afterwards on a case's own stream follows the batch. */
int dsmc_batch_step(DsmcBatch* b, int32_t nsteps);

/* The stream the batch graph runs on (a cudaStream_t), and a wait for it
 * that also reports device-side errors of the cases. */
void* dsmc_batch_stream(DsmcBatch* b);
int dsmc_batch_sync(DsmcBatch* b);

#ifdef __cplusplus
}
#endif
#endif /* DSMC_GPU_H */
