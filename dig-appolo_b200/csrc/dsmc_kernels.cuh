// Kernel argument blocks and launch wrappers shared by the engine.
#pragma once

#include "dsmc_device.cuh"

namespace dsmc {

template <typename Real>
struct PBuf {
    Real* x[3];
    Real* v[3];
    Real* ir;
    int* cell;
};

// Device-resident step control (read by kernels, so captured graphs replay
// with the current values).
struct StepCtl {
    int istep;
    int nLive;        // particles in the current buffer
    int nInj;         // particles injected this step (appended after nLive)
    int nNext;        // particles after the sort
    int capacity;
    int moveCursor;   // list entries handed out by the tracing pass of the move (reset before each move)
    int moveList;     // particles the stay pass leaves to the tracing pass (reset before each move)
    int pad[1];
};

struct DevPatches {
    int npatch, ngroup;
    const int* groupStart;     // [ngroup+1] into patch arrays (patches grouped by cell)
    const int* cell;           // [npatch]
    const int* edge;           // [npatch]
    const int* triTag;         // [npatch]
    const double* geom;        // [npatch*9] p0, e10, e20
    const double* rot;         // [npatch*9] rotation of -normal
    const double* gas;         // [npatch*8] snp, fs1, fs2, stp1, stp2, tN, sqrt(tN), QA
    const double* addBase;     // [npatch]
    int* count;                // [npatch] this step
    int* start;                // [npatch] exclusive scan
};

template <typename Real>
struct StepArgs {
    DevMesh M;
    DevConsts C;
    DevPatches P;
    PBuf<Real> A;             // current buffer (source of the step)
    PBuf<Real> B;             // next buffer (sorted output)
    const int* startA;        // [ncell+1] layout of A
    int* startB;              // [ncell+1] layout of B
    int* rank;                // [cap] packed slot<<24 | rank
    int* idx;                 // [cap] sorted source indices
    int* countSlot;           // [ncell*8]
    int* scanPartial;         // [kScanBlocks]
    double* crmax;            // [ncell]
    double* remColl;          // [ncell]
    double* remInj;           // [ncell]
    double* acc;              // [ncell*54]: stepsum, steady, stepinter (18 each)
    double* record;           // [ncell*18]
    double* local;            // [ncell*18]
    double* finalRecord;      // [ncell*18]
    double* stepMom;          // [ncell*18] or nullptr
    unsigned char* sparseState;
    int* sparseAccum;
    double* windowSamples;
    char* windowValid;
    double* wallTally;        // [nwall*6]
    StepCtl* ctl;
    unsigned long long* counters;
    int* cellPairs;           // [ncell] candidate pair count of the step (classify pass)
    double* cellCons;         // [ncell] majorant term of the pair count (classify pass)
    int* cellList;            // [2*ncell] work lists of the cell pass
    int4* cellItem;           // [ncell] huge / large items at their list slot: cell, start, count, pairs
    double2* cellItemC;       // [ncell] the same items' majorant term and crmax
    int* cellWork;            // [8] list lengths and hand-out counters of the cell pass
    int* errorWord;
};

constexpr int kScanBlocks = 296;

// Launch shapes of the step's kernels. Every kernel loops over its work
// (grid-stride or dynamic hand-out) and draws from counter-based streams, so
// results do not depend on these; only the speed does.
struct LaunchShape {
    int smCount = 148;
    int moveThreads = 256;        // threads per block of the move kernel: 128 or 256
    int moveBlocksPerSm = 8;      // move grid = smCount x this
    int sortBlocksPerSm = 16;     // rank, scatter, gather grids = smCount x this
    int collideBlocksPerSm = 32;  // collide grid cap per SM (at most the resident blocks)
    int stayPerThread = 4;        // particles per thread of the move's stay pass: 1, 2 or 4
};

template <typename Real> void launch_inject(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s);
template <typename Real> void launch_move(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s);
template <typename Real> void launch_sort(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s);
template <typename Real> void launch_collide(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s);
template <typename Real> void launch_sample(const StepArgs<Real>& a, bool pre, const LaunchShape& L, cudaStream_t s);
void launch_bump_istep(StepCtl* ctl, cudaStream_t s);

// Freestream of the initial fill, normalised like the particle state.
struct FillParams {
    double u[3];      // drift
    double sig;       // thermal spread per component, sqrt(T/2)
    double tN;        // temperature (rotational energy mean tN/2)
    uint32_t keyLo, keyHi;
};
template <typename Real>
void launch_fill(const StepArgs<Real>& a, const FillParams& f, const int* tetFirst, const LaunchShape& L, cudaStream_t s);
// exclusive scan of the countSlot rows into start[0..ncell], total into ctl->nNext
void launch_scan_counts(const int* countSlot, int ncell, int* partial, int* start, StepCtl* ctl, cudaStream_t s);

// GSIS particle update (molecular_velocity_change, src/ProcessGSIS.cpp:2239-2366)
struct GsisArgs {
    const double* ns;                // [ncell*6] density / n_ref, u (3), T, Tr
    const unsigned char* accepted;   // [ncell] or nullptr (acceptance gate off)
    int firstNan;                    // cells from this one on are left untouched
    uint32_t keyLo, keyHi;
    uint32_t purpose;                // kPurposeGsis | epoch << 8
    int* flag;                       // [ncell] 1: the cell is updated
    unsigned long long* tally;       // [4] cells updated, cells skipped, particles added, removed
};
// target counts into the countSlot rows and their scan into startB / ctl->nNext
template <typename Real> void launch_gsis_count(const StepArgs<Real>& a, const GsisArgs& g, cudaStream_t s);
// B from A: kept, copied, sampled and deleted particles, then the per-cell linear map
template <typename Real> void launch_gsis_rebuild(const StepArgs<Real>& a, const GsisArgs& g, const LaunchShape& L,
                                                  cudaStream_t s);
// Particle upload from cell-major host arrays: flags bit 0 a cell id outside
// [0, ncell), bit 1 a cell id smaller than its predecessor's; when neither
// is set, start[0..ncell] holds each cell's first slot.
void launch_upload_check(const int* cell, int n, int ncell, int* flags, int* start, cudaStream_t s);
// out[i] = (float)(in[i] - center[cell[i] * 3 + comp]) for comp < 3, else (float)in[i]
void launch_upload_convert(const double* in, const int* cell, const double* center, int comp, float* out, int n,
                           cudaStream_t s);
template <typename Real> cudaError_t prepare_kernels();
void launch_macro(const DevMesh& M, const DevConsts& C, const double* acc, int set, double count,
                  double* out, int ncell, cudaStream_t s);
template <typename Real>
void launch_trace_check(const DevMesh& M, const DevConsts& C, int n, const Real* px, const Real* py,
                        const Real* pz, const Real* vx, const Real* vy, const Real* vz,
                        const double* dt, const int* cell, int stopAtWall, int* oCell, int* oIfout,
                        int* oFace, int* oTri, int* oNcross, int* oLast, Real* ox, Real* oy, Real* oz,
                        Real* ovx, Real* ovy, Real* ovz, double* odt, unsigned long long* counters,
                        cudaStream_t s);

}  // namespace dsmc
