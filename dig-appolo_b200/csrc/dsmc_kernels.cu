// The DSMC step kernels.
//
//   inject   preprocesseffquad (src/ProcessDSMC.cpp:2556-2570): per-cell
//            inflow counts with the reference's remainder carry, scan,
//            per-patch particle generation + trace for r*dt.
//   move     advection (src/ProcessDSMC.cpp:1946-2017): lanes trace
//            particles for dtime through the mesh, refilled from warp
//            chunks as their particles finish.
//   sort     cache2chain (src/ProcessDSMC.cpp:2030-2135): deterministic
//            counting sort. rank (warp per source cell: arrival slot and rank
//            from warp ballots; multi-hop and injected arrivals through
//            warp-aggregated atomics), scan, scatter of source indices, the
//            far arrivals put in source order, gather of the particles.
//   collide  collisionDSMC (src/ProcessDSMC.cpp:2621-2744): cells classed
//            by size; NTC candidate pairs in sequence per cell (claims keep
//            the reference's pair order), accepted pairs run together.
//   sample   statistic_macro (src/ProcessDSMC.cpp:2757-2861): the
//            18-moment sums of each cell in particle order.
#include <climits>
#include <cstddef>
#include <type_traits>

#include "dsmc_kernels.cuh"
#include "dsmc_macro.cuh"

namespace dsmc {

constexpr unsigned kFull = 0xffffffffu;


// Particle positions between HBM and the trace's FP64 registers: the FP64
// path stores absolute FP64; the mixed path stores FP32 offsets from the
// centre of the particle's cell (widened as centre + offset, stored as the
// FP32 rounding of position - centre).
template <typename Real>
__device__ __forceinline__ void load_position(const DevMesh& M, const PBuf<Real>& B, int i, int cell, PRegs<Real>& p)
{
    if constexpr (sizeof(Real) == 8) {
        p.x[0] = B.x[0][i]; p.x[1] = B.x[1][i]; p.x[2] = B.x[2][i];
    } else {
        const double* cc = M.cellCenter + (size_t)cell * 3;
        p.x[0] = da(cc[0], (double)B.x[0][i]);
        p.x[1] = da(cc[1], (double)B.x[1][i]);
        p.x[2] = da(cc[2], (double)B.x[2][i]);
    }
}

template <typename Real>
__device__ __forceinline__ void store_position(const DevMesh& M, const PBuf<Real>& B, int i, int cell,
                                               const PRegs<Real>& p)
{
    if constexpr (sizeof(Real) == 8) {
        B.x[0][i] = p.x[0]; B.x[1][i] = p.x[1]; B.x[2][i] = p.x[2];
    } else {
        if (cell < 0 || cell >= M.ncell) return;   // removed: the slot is not read again
        const double* cc = M.cellCenter + (size_t)cell * 3;
        B.x[0][i] = (float)ds(p.x[0], cc[0]);
        B.x[1][i] = (float)ds(p.x[1], cc[1]);
        B.x[2][i] = (float)ds(p.x[2], cc[2]);
    }
}

// ===========================================================================
// inject
// ===========================================================================
__global__ void inject_count_kernel(DevPatches P, double* remInj)
{
    for (int g = blockIdx.x * blockDim.x + threadIdx.x; g < P.ngroup; g += gridDim.x * blockDim.x) {
        const int b = P.groupStart[g];
        const int e = P.groupStart[g + 1];
        const int cell = P.cell[b];
        double rem = remInj[cell];
        // computeBoundaryInsertCount, src/ProcessDSMC.cpp:2398-2402
        for (int p = b; p < e; ++p) {
            const double addNum = da(P.addBase[p], rem);
            const double fl = floor(addNum);
            const int n = (int)fl;
            rem = ds(addNum, (double)n);
            P.count[p] = n;
        }
        remInj[cell] = rem;
    }
}

__global__ void __launch_bounds__(1024) inject_scan_kernel(DevPatches P, StepCtl* ctl, unsigned long long* counters)
{
    __shared__ int warpSum[32];
    __shared__ int carry;
    const int tid = threadIdx.x;
    const int lane = tid & 31, wid = tid >> 5;
    const int room = ctl->capacity - ctl->nLive;
    if (tid == 0) carry = 0;
    long long over = 0;
    __syncthreads();
    for (int base = 0; base < P.npatch; base += blockDim.x) {
        const int i = base + tid;
        const int v = (i < P.npatch) ? P.count[i] : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSum[wid] = x;
        __syncthreads();
        if (wid == 0) {
            int w = (lane < (int)(blockDim.x >> 5)) ? warpSum[lane] : 0;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int y = __shfl_up_sync(kFull, w, o);
                if (lane >= o) w += y;
            }
            warpSum[lane] = w;
        }
        __syncthreads();
        const int incl = x + (wid > 0 ? warpSum[wid - 1] : 0);
        const int start = carry + incl - v;
        if (i < P.npatch) {
            P.start[i] = start;
            int allowed = room - start;
            allowed = allowed < 0 ? 0 : (allowed > v ? v : allowed);
            if (allowed < v) {
                over += v - allowed;
                P.count[i] = allowed;
            }
        }
        __syncthreads();
        if (tid == blockDim.x - 1) carry += incl;
        __syncthreads();
    }
    if (over) atomicAdd(counters + C_OVERFLOW, (unsigned long long)over);
    __syncthreads();
    if (tid == 0) {
        const int m = carry < room ? carry : (room > 0 ? room : 0);
        ctl->nInj = m;
        atomicAdd(counters + C_INJECTED, (unsigned long long)m);
    }
}

// sampleBoundaryParticle, src/ProcessDSMC.cpp:2416-2458: normal speed by
// acceptance-rejection against the fs1/fs2 envelope, tangential components by
// Box-Muller, rotational energy -ln(r) T / 2, all in the patch frame.
__device__ __forceinline__ void sample_inflow_velocity(const double* gas, const double* R, Stream& rs,
                                                       double v[3], double& ir, int* errorWord)
{
    const double snp = gas[0], fs1 = gas[1], fs2 = gas[2], stp1 = gas[3], stp2 = gas[4];
    const double tN = gas[5], sq = gas[6], QA = gas[7];
    double vzr = 0.0, vza = 0.0;
    for (int outer = 0;; ++outer) {
        for (int inner = 0;; ++inner) {
            const double r = rs.uniform64();
            vzr = (-QA + 2.0 * QA * r) * sq;
            vza = vzr / sq + snp;
            if (vza > 0) break;
            if (inner > (1 << 20)) { atomicOr(errorWord, kErrRejectLoop); vza = 1e-3; break; }
        }
        const double vzn = vzr / sq;
        const double pp = (2.0 * vza / fs1) * exp(fs2 - vzn * vzn);
        if (rs.uniform64() < pp) break;
        if (outer > (1 << 20)) { atomicOr(errorWord, kErrRejectLoop); break; }
    }
    const double r = rs.uniform64();
    const double th = rs.uniform64();
    double s, c;
    sincospi(2.0 * th, &s, &c);
    const double a = sqrt(-log(r));
    const double vxa = (a * s + stp1) * sq;
    const double vya = (a * c + stp2) * sq;
    vza *= sq;
    v[0] = R[0] * vxa + R[1] * vya + R[2] * vza;
    v[1] = R[3] * vxa + R[4] * vya + R[5] * vza;
    v[2] = R[6] * vxa + R[7] * vya + R[8] * vza;
    ir = -log(rs.uniform64()) * tN * 0.5;
}

// One thread per injected particle; its patch is found by binary search in
// the exclusive scan of the per-patch counts (slots of one patch are
// consecutive, so a warp mostly works on one patch).
template <typename Real>
__global__ void __launch_bounds__(128) inject_gen_kernel(StepArgs<Real> a)
{
    const int istep = a.ctl->istep;
    const int nLive = a.ctl->nLive;
    const int m = a.ctl->nInj;
    const int np = a.P.npatch;
    TraceCounts cnt{};
    for (int slot = blockIdx.x * blockDim.x + threadIdx.x; slot < m; slot += gridDim.x * blockDim.x) {
        int lo = 0, hi = np - 1;          // last patch with start <= slot
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (a.P.start[mid] <= slot) lo = mid; else hi = mid - 1;
        }
        const int p = lo;
        const int pcell = a.P.cell[p];
        const int pedge = a.P.edge[p];
        const int ptag = a.P.triTag[p];
        const double* G = a.P.geom + (size_t)p * 9;
        const double* R = a.P.rot + (size_t)p * 9;
        const double* gas = a.P.gas + (size_t)p * 8;
        const int gi = nLive + slot;
        Stream rs;
        rs.init((uint32_t)gi, (uint32_t)istep, kPurposeInject, a.C.seedLo, a.C.seedHi);
        double u = rs.uniform64(), w = rs.uniform64();
        if (u + w > 1.0) { u = 1.0 - u; w = 1.0 - w; }
        double pos[3];
        // p0 + u e10 + v e20 (src/ProcessDSMC.cpp:2524-2526), unfused
        for (int d = 0; d < 3; ++d) pos[d] = da(da(G[d], dm(u, G[3 + d])), dm(w, G[6 + d]));
        double vel[3], irv;
        sample_inflow_velocity(gas, R, rs, vel, irv, a.errorWord);
        double dtleft = rs.uniform64() * a.C.dtime;
        PRegs<Real> pr;
        int cell = pcell;
        for (int d = 0; d < 3; ++d) pr.x[d] = pos[d];
        for (int d = 0; d < 3; ++d) pr.v[d] = (Real)vel[d];
        pr.ir = (Real)irv;
        const int out = trace_particle<Real>(a.M, a.C, pr, cell, pedge, ptag, dtleft, rs, istep,
                                             a.wallTally, cnt, false, nullptr);
        store_position(a.M, a.A, gi, cell, pr);
        a.A.v[0][gi] = pr.v[0]; a.A.v[1][gi] = pr.v[1]; a.A.v[2][gi] = pr.v[2];
        a.A.ir[gi] = pr.ir;
        a.A.cell[gi] = (out >= 0) ? cell : -1;
    }
    flush_counts(a.counters, cnt);
}

template <typename Real>
void launch_inject(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s)
{
    if (a.P.npatch == 0) {
        cudaMemsetAsync(&a.ctl->nInj, 0, sizeof(int), s);
        return;
    }
    const int gCount = (a.P.ngroup + 127) / 128;
    inject_count_kernel<<<gCount > 0 ? gCount : 1, 128, 0, s>>>(a.P, a.remInj);
    inject_scan_kernel<<<1, 1024, 0, s>>>(a.P, a.ctl, a.counters);
    inject_gen_kernel<Real><<<L.smCount * 8, 128, 0, s>>>(a);
}

// ===========================================================================
// move
// ===========================================================================
// Two passes over the particles of the step.
//
// Stay pass (move_stay_kernel): one thread per particle, in slot order
// (coalesced loads, the particles of a cell next to each other, so a warp
// reads few cells' face records). Most particles stay in their cell for the
// whole step; where the first exit search settles that (stays_for_the_step)
// the particle is advanced and stored right there. The others are appended
// to a work list (warp-aggregated, in the sort's rank array, which is free
// until the sort), with their state copied to the same positions of the
// other particle buffer (free until the sort too): the tracing pass then
// reads its particles in list order instead of gathering them from sparse
// slots (move 2.18 -> 2.08 ms). (Handing the crossing that search settled
// to the tracing pass as well was measured slower: 2.37 against 2.17 ms.)
//
// Tracing pass (move_kernel): the listed particles, traced from their start
// by trace_step. Warps claim chunks of 128 list entries from a cursor in
// the step control block (one atomic per chunk), and a lane whose particle
// has finished writes it back and takes the next particle of the chunk, so
// the lanes keep doing exit searches instead of waiting for the warp's
// longest trace. Three resident 256-thread blocks per SM (registers capped
// at 85): the trace is bound by dependent loads, so occupancy pays more than
// the few registers it spills to L1.
//
// Each particle runs the same code with its own random stream (particle
// index, step), and the stay pass takes exactly the decision the trace's
// first search takes, so results do not depend on the split, the list
// order, or which lane or warp traces a particle.
constexpr int kMoveChunk = 128;

// K particles per thread (K x 256 consecutive slots per block and round):
// the loads of all K are issued before the first decision.
template <typename Real, int K>
__global__ void __launch_bounds__(256) move_stay_kernel(StepArgs<Real> a)
{
    const int n = a.ctl->nLive;
    const double dt = a.C.dtime;
    const int lane = threadIdx.x & 31;
    const int tile = K * (int)blockDim.x;
    for (int base = blockIdx.x * tile; base < n; base += gridDim.x * tile) {
        int cell[K];
        Real xs[K][3];
        PRegs<Real> p[K];
        // the slot's own loads first, all of them independent of each other
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = base + k * (int)blockDim.x + (int)threadIdx.x;
            if (i < n) {
                cell[k] = a.A.cell[i];
                xs[k][0] = a.A.x[0][i]; xs[k][1] = a.A.x[1][i]; xs[k][2] = a.A.x[2][i];
                p[k].v[0] = a.A.v[0][i]; p[k].v[1] = a.A.v[1][i]; p[k].v[2] = a.A.v[2][i];
            } else {
                cell[k] = -1;
            }
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int i = base + k * (int)blockDim.x + (int)threadIdx.x;
            bool defer = false;
            if (cell[k] >= 0) {
                // the position as load_position widens it
                if constexpr (sizeof(Real) == 8) {
                    p[k].x[0] = xs[k][0]; p[k].x[1] = xs[k][1]; p[k].x[2] = xs[k][2];
                } else {
                    const double* cc = a.M.cellCenter + (size_t)cell[k] * 3;
                    p[k].x[0] = da(cc[0], (double)xs[k][0]);
                    p[k].x[1] = da(cc[1], (double)xs[k][1]);
                    p[k].x[2] = da(cc[2], (double)xs[k][2]);
                }
                if (stays_for_the_step<Real>(a.M, cell[k], p[k], dt)) {
                    advance(p[k], dt);
                    store_position(a.M, a.A, i, cell[k], p[k]);
                } else {
                    defer = true;
                }
            }
            const unsigned m = __ballot_sync(kFull, defer);
            if (m) {
                int at = 0;
                if (lane == 0) at = atomicAdd(&a.ctl->moveList, __popc(m));
                at = __shfl_sync(kFull, at, 0);
                if (defer) {
                    // the entry: the slot, and the particle's state in the
                    // other buffer (free until the sort) at the same
                    // position, so the tracing pass reads it in list order
                    const int j = at + __popc(m & ((1u << lane) - 1u));
                    a.rank[j] = i;
                    a.B.cell[j] = cell[k];
                    a.B.x[0][j] = xs[k][0]; a.B.x[1][j] = xs[k][1]; a.B.x[2][j] = xs[k][2];
                    a.B.v[0][j] = p[k].v[0]; a.B.v[1][j] = p[k].v[1]; a.B.v[2][j] = p[k].v[2];
                    a.B.ir[j] = a.A.ir[i];
                }
            }
        }
    }
}

template <typename Real>
__global__ void __launch_bounds__(256, 3) move_kernel(StepArgs<Real> a)
{
    const int istep = a.ctl->istep;
    const int n = a.ctl->moveList;
    const int* __restrict__ list = a.rank;
    const int lane = threadIdx.x & 31;
    const unsigned lower = (1u << lane) - 1u;
    TraceCounts cnt{};
    const double dt0 = a.C.dtime;
    int chunkNext = 0, chunkEnd = 0;   // this warp's chunk (warp-uniform)
    bool exhausted = false;            // warp-uniform
    int i = -1;                        // this lane's particle
    PRegs<Real> p;
    int cell = 0;
    double dtleft = 0;
    TraceState st;
    // the particle's wall draws; the mixed path's in one register (drawn a
    // re-emission at a time, from block 0)
    using Rng = typename std::conditional<sizeof(Real) == 4, BlockStream, Stream>::type;
    Rng rs;
    uint32_t wallBefore = 0;
    for (;;) {
        unsigned want = __ballot_sync(kFull, i < 0);
        while (want && !exhausted) {
            if (chunkNext >= chunkEnd) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&a.ctl->moveCursor, kMoveChunk);
                base = __shfl_sync(kFull, base, 0);
                if (base >= n) {
                    exhausted = true;
                    break;
                }
                chunkNext = base;
                chunkEnd = min(base + kMoveChunk, n);
            }
            const int take = min(chunkEnd - chunkNext, __popc(want));
            const bool mine = ((want >> lane) & 1u) && __popc(want & lower) < take;
            if (mine) {
                // the entry's slot and state, as the stay pass wrote them
                const int j = chunkNext + __popc(want & lower);
                i = list[j];
                cell = a.B.cell[j];
                load_position(a.M, a.B, j, cell, p);
                p.v[0] = a.B.v[0][j]; p.v[1] = a.B.v[1][j]; p.v[2] = a.B.v[2][j];
                p.ir = a.B.ir[j];
                if constexpr (sizeof(Real) == 4) rs.init((uint32_t)i, (uint32_t)istep, kPurposeWall);
                else rs.init((uint32_t)i, (uint32_t)istep, kPurposeWall, a.C.seedLo, a.C.seedHi);
                dtleft = dt0;
                st.begin(-1, -1);
                wallBefore = cnt.wall;
            }
            chunkNext += take;
            want &= ~__ballot_sync(kFull, mine);
        }
        const bool active = i >= 0;
        if (!__any_sync(kFull, active)) break;
        if (active && trace_step<Real, Rng>(a.M, a.C, p, cell, dtleft, st, rs, istep, a.wallTally, cnt, false, nullptr)) {
            if (st.ifout >= 0) {
                store_position(a.M, a.A, i, cell, p);
                if (cnt.wall != wallBefore) {
                    a.A.v[0][i] = p.v[0]; a.A.v[1][i] = p.v[1]; a.A.v[2][i] = p.v[2];
                    a.A.ir[i] = p.ir;
                }
                a.A.cell[i] = cell;
            } else {
                a.A.cell[i] = -1;
            }
            i = -1;
        }
    }
    flush_counts(a.counters, cnt);
}

// resident blocks per SM of the stay pass (1, 2, 4 particles per thread),
// set by prepare_kernels
template <typename Real>
struct StayOcc {
    static int blocks[3];
};
template <typename Real>
int StayOcc<Real>::blocks[3] = {4, 4, 4};

template <typename Real>
void launch_move(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s)
{
    static_assert(offsetof(StepCtl, moveList) == offsetof(StepCtl, moveCursor) + sizeof(int),
                  "the move's cursor and list count are reset together");
    cudaMemsetAsync(&a.ctl->moveCursor, 0, 2 * sizeof(int), s);
    // one wave: every block resident (the blocks split the slots evenly, so
    // a second, partial wave would run at a fraction of the occupancy)
    if (L.stayPerThread == 4)
        move_stay_kernel<Real, 4><<<L.smCount * StayOcc<Real>::blocks[2], 256, 0, s>>>(a);
    else if (L.stayPerThread == 2)
        move_stay_kernel<Real, 2><<<L.smCount * StayOcc<Real>::blocks[1], 256, 0, s>>>(a);
    else
        move_stay_kernel<Real, 1><<<L.smCount * StayOcc<Real>::blocks[0], 256, 0, s>>>(a);
    move_kernel<Real><<<L.smCount * L.moveBlocksPerSm, L.moveThreads, 0, s>>>(a);
}

// advance the step counter on the device (batched steps, where the graph
// carries no host-written step number)
__global__ void bump_istep_kernel(StepCtl* ctl) { ctl->istep += 1; }

void launch_bump_istep(StepCtl* ctl, cudaStream_t s) { bump_istep_kernel<<<1, 1, 0, s>>>(ctl); }

// ===========================================================================
// sort: rank, scan, scatter
// ===========================================================================
template <typename Real>
__global__ void __launch_bounds__(256) rank_kernel(StepArgs<Real> a)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const int ncell = a.M.ncell;
    const unsigned lt = (1u << lane) - 1u;
    for (int s = warp; s < ncell; s += nwarps) {
        const int b = a.startA[s];
        const int e = a.startA[s + 1];
        const int nbL = (lane < 6) ? a.M.cell2cell[(size_t)s * 6 + lane] : -1;
        const int rvL = (lane < 6) ? (int)a.M.revSlot[(size_t)s * 6 + lane] : -1;
        int nbr[6], slotQ[7], runQ[7];
        slotQ[0] = 0;
        runQ[0] = 0;
#pragma unroll
        for (int j = 0; j < 6; ++j) {
            nbr[j] = __shfl_sync(kFull, nbL, j);
            slotQ[j + 1] = __shfl_sync(kFull, rvL, j) + 1;
            runQ[j + 1] = 0;
        }
        // the cell ids of up to 128 particles loaded first, then ranked 32 at
        // a time
        for (int base4 = b; base4 < e; base4 += 128) {
            int dq[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int i = base4 + 32 * u + lane;
                dq[u] = i < e ? a.A.cell[i] : -1;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int base = base4 + 32 * u;
                if (base >= e) break;
                const int i = base + lane;
                const bool valid = i < e;
                const int d = dq[u];
                int q = -1;
                if (d >= 0) {
                    if (d == s) q = 0;
                    else {
#pragma unroll
                        for (int j = 5; j >= 0; --j)
                            if (d == nbr[j]) q = j + 1;
                    }
                }
                int packed = -1;
#pragma unroll
                for (int qq = 0; qq < 7; ++qq) {
                    const unsigned m = __ballot_sync(kFull, q == qq);
                    if (q == qq) packed = (slotQ[qq] << 24) | (runQ[qq] + __popc(m & lt));
                    runQ[qq] += __popc(m);
                }
                // multi-cell hops (a few percent): a slot each; their order is
                // made canonical after the scatter
                if (d >= 0 && q < 0) packed = (kFarSlot << 24) | atomicAdd(a.countSlot + (size_t)d * kSlots + kFarSlot, 1);
                if (valid) a.rank[i] = packed;
            }
        }
        int myRun = 0;
#pragma unroll
        for (int qq = 0; qq < 7; ++qq)
            if (lane == qq) myRun = runQ[qq];
        const int nbPrev = __shfl_up_sync(kFull, nbL, 1);
        const int rvPrev = __shfl_up_sync(kFull, rvL, 1);
        if (lane == 0) {
            a.countSlot[(size_t)s * kSlots] = myRun;
        } else if (lane <= 6) {
            if (nbPrev >= 0 && nbPrev < ncell && rvPrev >= 0) a.countSlot[(size_t)nbPrev * kSlots + rvPrev + 1] = myRun;
        }
    }
    // injected particles: all arrive through the far slot
    const int nLive = a.ctl->nLive;
    const int nTot = nLive + a.ctl->nInj;
    for (int base = nLive + warp * 32; base < nTot; base += nwarps * 32) {
        const int i = base + lane;
        const int d = (i < nTot) ? a.A.cell[i] : -1;
        const int key = d >= 0 ? d * kSlots + kFarSlot : -1;
        const int r = warp_claim(a.countSlot, key);
        if (i < nTot && d >= 0) a.rank[i] = (kFarSlot << 24) | r;
    }
}

__device__ __forceinline__ int row_total(const int* countSlot, int c)
{
    const int4 lo = *reinterpret_cast<const int4*>(countSlot + (size_t)c * kSlots);
    const int4 hi = *reinterpret_cast<const int4*>(countSlot + (size_t)c * kSlots + 4);
    return lo.x + lo.y + lo.z + lo.w + hi.x + hi.y + hi.z + hi.w;
}

__device__ __forceinline__ int block_sum(int v, int* sh)
{
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    if (lane == 0) sh[wid] = v;
    __syncthreads();
    int t = 0;
    if (threadIdx.x == 0)
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    __syncthreads();
    if (threadIdx.x == 0) sh[0] = t;
    __syncthreads();
    const int r = sh[0];
    __syncthreads();
    return r;
}

__global__ void __launch_bounds__(256) scan_partial_kernel(const int* countSlot, int ncell, int* partial)
{
    __shared__ int sh[32];
    const int chunk = (ncell + gridDim.x - 1) / gridDim.x;
    const int b = blockIdx.x * chunk;
    const int e = min(ncell, b + chunk);
    int s = 0;
    for (int c = b + threadIdx.x; c < e; c += blockDim.x) s += row_total(countSlot, c);
    s = block_sum(s, sh);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

__global__ void __launch_bounds__(256) scan_final_kernel(const int* countSlot, int ncell, const int* partial,
                                                         int* start, StepCtl* ctl)
{
    __shared__ int sh[32];
    __shared__ int warpSum[8];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    int pre = 0;
    for (int k = threadIdx.x; k < (int)blockIdx.x; k += blockDim.x) pre += partial[k];
    int carry = block_sum(pre, sh);
    const int chunk = (ncell + gridDim.x - 1) / gridDim.x;
    const int b = blockIdx.x * chunk;
    const int e = min(ncell, b + chunk);
    for (int base = b; base < e; base += blockDim.x) {
        const int c = base + threadIdx.x;
        const int v = (c < e) ? row_total(countSlot, c) : 0;
        int x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(kFull, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warpSum[wid] = x;
        __syncthreads();
        int off = 0;
        for (int w = 0; w < wid; ++w) off += warpSum[w];
        int tileTotal = 0;
        for (int w = 0; w < 8; ++w) tileTotal += warpSum[w];
        if (c < e) start[c] = carry + off + x - v;
        __syncthreads();
        carry += tileTotal;
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) {
        start[ncell] = carry;
        ctl->nNext = carry;
    }
}

template <typename Real>
__global__ void __launch_bounds__(256) scatter_kernel(StepArgs<Real> a)
{
    // four particles per thread, their loads issued before their stores
    constexpr int U = 4;
    const int nTot = a.ctl->nLive + a.ctl->nInj;
    const int stride = gridDim.x * blockDim.x;
    for (int i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < nTot; i0 += U * stride) {
        int d[U], packed[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int i = i0 + u * stride;
            d[u] = i < nTot ? a.A.cell[i] : -1;
            packed[u] = i < nTot ? a.rank[i] : 0;
        }
        int4 lo[U], hi[U];
        int s0[U], s1[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (d[u] < 0) continue;
            lo[u] = *reinterpret_cast<const int4*>(a.countSlot + (size_t)d[u] * kSlots);
            hi[u] = *reinterpret_cast<const int4*>(a.countSlot + (size_t)d[u] * kSlots + 4);
            s0[u] = a.startB[d[u]];
            s1[u] = a.startB[d[u] + 1];
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (d[u] < 0) continue;
            const int slot = packed[u] >> 24;
            int base = s0[u] + (packed[u] & 0xFFFFFF);
            if (slot > 0) base += lo[u].x;
            if (slot > 1) base += lo[u].y;
            if (slot > 2) base += lo[u].z;
            if (slot > 3) base += lo[u].w;
            if (slot > 4) base += hi[u].x;
            if (slot > 5) base += hi[u].y;
            if (slot > 6) base += hi[u].z;
            if (base < s0[u] || base >= s1[u]) {   // self-check: slot counts inconsistent
                atomicOr(a.errorWord, kErrSortIndex);
                continue;
            }
            a.idx[base] = i0 + u * stride;
            a.B.cell[base] = d[u];
        }
    }
}

// Ascending bitonic sort of 32*K keys held K per lane (element e of lane l is
// position e*32 + l). Unused slots hold 0xffffffff.
template <int K>
__device__ __forceinline__ void warp_bitonic(uint32_t (&a)[K])
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int k = 2; k <= 32 * K; k <<= 1) {
#pragma unroll
        for (int j = k >> 1; j > 0; j >>= 1) {
            if (j >= 32) {
                const int je = j >> 5;
#pragma unroll
                for (int e = 0; e < K; ++e) {
                    const int e2 = e ^ je;
                    if (e2 > e) {
                        const bool asc = (((e << 5) | lane) & k) == 0;
                        const uint32_t lo = min(a[e], a[e2]), hi = max(a[e], a[e2]);
                        a[e] = asc ? lo : hi;
                        a[e2] = asc ? hi : lo;
                    }
                }
            } else {
#pragma unroll
                for (int e = 0; e < K; ++e) {
                    const uint32_t o = __shfl_xor_sync(kFull, a[e], j);
                    const bool asc = (((e << 5) | lane) & k) == 0;
                    const bool lower = (lane & j) == 0;
                    a[e] = (lower == asc) ? min(a[e], o) : max(a[e], o);
                }
            }
        }
    }
}

template <int K>
__device__ __forceinline__ void sort_far_warp(int* seg, int m)
{
    const int lane = threadIdx.x & 31;
    uint32_t v[K];
#pragma unroll
    for (int e = 0; e < K; ++e) {
        const int p = e * 32 + lane;
        v[e] = (p < m) ? (uint32_t)seg[p] : 0xffffffffu;
    }
    warp_bitonic<K>(v);
    __syncwarp();
#pragma unroll
    for (int e = 0; e < K; ++e) {
        const int p = e * 32 + lane;
        if (p < m) seg[p] = (int)v[e];
    }
    __syncwarp();
}

// Canonical order of a cell's far-slot arrivals: ascending source index.
// tmp is a scratch range of the same length (the output buffer's cell ids
// at those positions, written later by the gather).
__device__ void sort_far(int* seg, int m, int* tmp)
{
    const int lane = threadIdx.x & 31;
    if (m <= 1) return;
    if (m <= 32) {
        sort_far_warp<1>(seg, m);
    } else if (m <= 512) {
        sort_far_warp<16>(seg, m);
    } else {
        // rank counting: O(m^2 / 32), for the rare very large far segments
        for (int e = lane; e < m; e += 32) tmp[e] = seg[e];
        __syncwarp();
        for (int e = lane; e < m; e += 32) {
            const int v = tmp[e];
            int r = 0;
            for (int f = 0; f < m; ++f) r += tmp[f] < v;
            seg[r] = v;
        }
        __syncwarp();
    }
}

// Canonical order of every cell's far-slot arrivals: ascending source
// index; the far counts are cleared for the next step's rank pass. Each
// lane takes one cell: a segment of up to kLaneSort arrivals (the common
// case: multi-cell hops and injected particles are some tens per cell at
// most) is insertion-sorted in the lane's own shared-memory row; longer
// ones by the whole warp, whose output cell ids serve as scratch for very
// long ones and are restored.
constexpr int kLaneSort = 32;
constexpr int kFarsortThreads = 256;

__global__ void __launch_bounds__(kFarsortThreads) farsort_kernel(int* countSlot, const int* startB, int* idx,
                                                                  int* cellB, int ncell)
{
    __shared__ int rows[kFarsortThreads][kLaneSort + 1];
    int* row = rows[threadIdx.x];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int base = warp * 32; base < ncell; base += nwarps * 32) {
        const int c = base + lane;
        int far = 0;
        if (c < ncell) {
            far = countSlot[(size_t)c * kSlots + kFarSlot];
            if (far) countSlot[(size_t)c * kSlots + kFarSlot] = 0;
        }
        if (far >= 2 && far <= kLaneSort) {
            int* seg = idx + startB[c + 1] - far;
            for (int k = 0; k < far; ++k) row[k] = seg[k];
            for (int k = 1; k < far; ++k) {
                const int v = row[k];
                int j = k - 1;
                while (j >= 0 && row[j] > v) {
                    row[j + 1] = row[j];
                    --j;
                }
                row[j + 1] = v;
            }
            for (int k = 0; k < far; ++k) seg[k] = row[k];
        }
        for (unsigned m = __ballot_sync(kFull, far > kLaneSort); m; m &= m - 1) {
            const int l = __ffs(m) - 1;
            const int cl = base + l;
            const int f = __shfl_sync(kFull, far, l);
            const int e = startB[cl + 1];
            sort_far(idx + e - f, f, cellB + e - f);
            if (f > 512) {
                for (int k = lane; k < f; k += 32) cellB[e - f + k] = cl;
                __syncwarp();
            }
        }
    }
}

// cache2chain's data move (src/ProcessDSMC.cpp:2030-2135): output slot o
// takes source particle idx[o]. Coalesced writes; the reads follow the
// source order of each arrival group.
template <typename Real>
__global__ void __launch_bounds__(256) gather_kernel(StepArgs<Real> a)
{
    // four output slots per thread, their loads issued before their stores
    constexpr int U = 4;
    const int n = a.ctl->nNext;
    const unsigned nSrc = (unsigned)(a.ctl->nLive + a.ctl->nInj);
    const int stride = gridDim.x * blockDim.x;
    for (int o0 = blockIdx.x * blockDim.x + threadIdx.x; o0 < n; o0 += U * stride) {
        int src[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int o = o0 + u * stride;
            src[u] = o < n ? a.idx[o] : -1;
        }
        Real x[U], y[U], z[U], vx[U], vy[U], vz[U], ir[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int o = o0 + u * stride;
            if (o < n && (unsigned)src[u] < nSrc) {
                const int i = src[u];
                x[u] = a.A.x[0][i]; y[u] = a.A.x[1][i]; z[u] = a.A.x[2][i];
                vx[u] = a.A.v[0][i]; vy[u] = a.A.v[1][i]; vz[u] = a.A.v[2][i];
                ir[u] = a.A.ir[i];
            }
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int o = o0 + u * stride;
            if (o >= n) continue;
            if ((unsigned)src[u] >= nSrc) {   // self-check: never index outside the source
                atomicOr(a.errorWord, kErrSortIndex);
                continue;
            }
            a.B.x[0][o] = x[u]; a.B.x[1][o] = y[u]; a.B.x[2][o] = z[u];
            a.B.v[0][o] = vx[u]; a.B.v[1][o] = vy[u]; a.B.v[2][o] = vz[u];
            a.B.ir[o] = ir[u];
        }
    }
}

template <typename Real>
void launch_sort(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s)
{
    const int g = L.smCount * L.sortBlocksPerSm;
    rank_kernel<Real><<<g, 256, 0, s>>>(a);
    scan_partial_kernel<<<kScanBlocks, 256, 0, s>>>(a.countSlot, a.M.ncell, a.scanPartial);
    scan_final_kernel<<<kScanBlocks, 256, 0, s>>>(a.countSlot, a.M.ncell, a.scanPartial, a.startB, a.ctl);
    scatter_kernel<Real><<<g, 256, 0, s>>>(a);
    farsort_kernel<<<L.smCount * 4, kFarsortThreads, 0, s>>>(a.countSlot, a.startB, a.idx, a.B.cell, a.M.ncell);
    gather_kernel<Real><<<g, 256, 0, s>>>(a);
}

// ===========================================================================
// collisions
// ===========================================================================

// collision_diameter, src/ProcessDSMC.cpp:2603-2608 (each operation rounded
// on its own, as the oracle and the reference's x86-64 build evaluate it)
__device__ __forceinline__ double collision_diameter(double cr, double prefactor, double eta)
{
    const double cr2 = dm(cr, cr);
    return dm(dm(cr, prefactor), pow(dd(1.0, cr2), eta));
}

// Division: IEEE in FP64 (the oracle's rounding), the fast reciprocal form
// in the FP32 path (operands here are far from the range limits).
__device__ __forceinline__ double qdiv(double x, double y) { return x / y; }
__device__ __forceinline__ float qdiv(float x, float y) { return __fdividef(x, y); }

// The random words of candidate pair j of cell c at step istep: Philox
// blocks n = 0, 1, ... of counter (c, istep, kPurposeCollide | j << 4),
// read in order as one stream. Block 0 is drawn when the pair is handed out
// (words 0, 1: the two particles; word 2 and in FP64 word 3: the acceptance
// variate); the rest only for accepted pairs, always at the same positions,
// so the lanes of a warp draw their blocks together.
// FP64 (the oracle's layout): block 1 = relaxation test and energy fraction
// of the first particle, block 2 the same for the second, block 3 = the
// deflection and azimuth variates, 53-bit uniforms from word pairs.
// FP32: word 3 of block 0 and word 0 of block 1 are the two relaxation
// tests, words 1 and 2 of block 1 the deflection and azimuth variates; a
// particle that relaxes (u <= P) takes u / P as its energy fraction, which
// given u <= P is again uniform on (0, 1], so one block less is drawn.
struct PairDraw {
    U4 b0;
    uint32_t c, istep, purpose;
    __device__ __forceinline__ U4 block(uint32_t n, const DevConsts& C) const
    {
        return philox4x32_10(U4{c, istep, purpose, n}, C.seedLo, C.seedHi);
    }
};

__device__ __forceinline__ PairDraw pair_draw(int c, int istep, int j, int n, const DevConsts& C, int& k1, int& k2)
{
    PairDraw d;
    d.c = (uint32_t)c; d.istep = (uint32_t)istep; d.purpose = kPurposeCollide | ((uint32_t)j << 4);
    d.b0 = d.block(0, C);
    k1 = (int)__umulhi(d.b0.x, (uint32_t)n);
    k2 = k1 + 1 + (int)__umulhi(d.b0.y, (uint32_t)(n - 1));
    if (k2 >= n) k2 -= n;
    return d;
}

// Square root: IEEE in FP64; in the FP32 path from the hardware reciprocal
// square root (a few ulp; the argument is a sum of squares, >= 0).
__device__ __forceinline__ double psqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float psqrt(float x) { return x > 0.0f ? x * rsqrtf(x) : 0.0f; }

// collisionVelocity, src/ProcessDSMC.cpp:2679-2744, on one candidate pair,
// in two halves: the acceptance test (pair_accept) and, for an accepted
// pair, the post-collision state (pair_execute). pair_execute recomputes the
// relative velocity from the same stored velocities, so the halves give the
// bits of the one-piece test-and-collide. Particle k of the cell is at
// vx[k * stride] (and likewise vy, vz, ir). w2, w3: words 2 and 3 of the
// pair's block 0. The FP64 branch rounds each operation on its own in the
// reference's evaluation order; the FP32 branch lets the compiler fuse.
template <typename Real>
__device__ __forceinline__ bool pair_accept(const Real* vx, const Real* vy, const Real* vz, int stride, int k1,
                                            int k2, uint32_t w2, uint32_t w3, const DevConsts& C, double consCrm,
                                            Real crm0, Real& crmLocal)
{
    k1 *= stride;
    k2 *= stride;
    if constexpr (sizeof(Real) == 8) {
        const double vr0 = ds(vx[k1], vx[k2]), vr1 = ds(vy[k1], vy[k2]), vr2 = ds(vz[k1], vz[k2]);
        const double cr = sqrt(da(da(dm(vr0, vr0), dm(vr1, vr1)), dm(vr2, vr2)));
        if (cr > crmLocal) crmLocal = cr;
        const double accept = dd(collision_diameter(dm(cr, C.vrms), C.cdPrefactor, C.eta), consCrm);
        return unit64(w2, w3) < accept;
    } else {
        const float vr0 = vx[k1] - vx[k2], vr1 = vy[k1] - vy[k2], vr2 = vz[k1] - vz[k2];
        const float cr = psqrt(vr0 * vr0 + vr1 * vr1 + vr2 * vr2);
        if (cr > crmLocal) crmLocal = cr;
        // ratio of the VHS sigma*c at cr and at crmax: (cr/crmax)^(1-2 eta)
        const float accept = exp2f(C.vhsExpF * __log2f(__fdividef(cr, crm0)));
        return unit32(w2) < accept;
    }
}

__device__ __forceinline__ void pair_execute_fp64(double* vx, double* vy, double* vz, double* ir, int k1, int k2,
                                                  const PairDraw& d, const DevConsts& C)
{
    const double v1x = vx[k1], v1y = vy[k1], v1z = vz[k1];
    const double v2x = vx[k2], v2y = vy[k2], v2z = vz[k2];
    const double vr0 = ds(v1x, v2x), vr1 = ds(v1y, v2y), vr2 = ds(v1z, v2z);
    const double cr2 = da(da(dm(vr0, vr0), dm(vr1, vr1)), dm(vr2, vr2));
    const double cr = sqrt(cr2);
    double preErt = dm(0.25, cr2);
    const U4 b1 = d.block(1, C), b2 = d.block(2, C), b3 = d.block(3, C);
    const double uRel[2] = {unit64(b1.x, b1.y), unit64(b2.x, b2.y)};
    const double rRel[2] = {unit64(b1.z, b1.w), unit64(b2.z, b2.w)};
    const double rChi = unit64(b3.x, b3.y), th = unit64(b3.z, b3.w);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        double* irp = (h == 0) ? &ir[k1] : &ir[k2];
        if (uRel[h] <= C.prelax) {
            const double preEr = *irp;
            const double postEr = dm(da(preErt, preEr), ds(1.0, pow(rRel[h], C.expLB)));
            *irp = postEr;
            preErt = ds(da(preErt, preEr), postEr);
        }
    }
    const double postVr = sqrt(dd(dm(2.0, preErt), 0.5));
    const double vc0 = dm(0.5, da(v1x, v2x)), vc1 = dm(0.5, da(v1y, v2y)), vc2 = dm(0.5, da(v1z, v2z));
    const double cosChi = ds(dm(2.0, pow(rChi, C.invAlpha)), 1.0);
    const double sinChi = sqrt(ds(1.0, dm(cosChi, cosChi)));
    const double ang = dm(6.283185307179586, th);   // 2 pi th
    const double sth = sin(ang), cth = cos(ang);
    const double vrp = sqrt(da(dm(vr1, vr1), dm(vr2, vr2)));
    const double scale = dd(postVr, cr > 1.0e-300 ? cr : 1.0e-300);
    const double vrpc = vrp > 1.0e-300 ? vrp : 1.0e-300;
    double r1, r2, r3;
    if (vrp < 1e-6) {
        r1 = dm(dm(scale, cosChi), vr0);
        r2 = dm(dm(dm(scale, sinChi), vr0), cth);
        r3 = dm(dm(dm(scale, sinChi), vr0), sth);
    } else {
        r1 = dm(scale, da(dm(cosChi, vr0), dm(dm(sinChi, sth), vrp)));
        r2 = dm(scale, da(dm(cosChi, vr1), dd(dm(sinChi, ds(dm(dm(cr, vr2), cth), dm(dm(vr0, vr1), sth))), vrpc)));
        r3 = dm(scale, ds(dm(cosChi, vr2), dd(dm(sinChi, da(dm(dm(cr, vr1), cth), dm(dm(vr0, vr2), sth))), vrpc)));
    }
    vx[k1] = da(vc0, dm(0.5, r1)); vy[k1] = da(vc1, dm(0.5, r2)); vz[k1] = da(vc2, dm(0.5, r3));
    vx[k2] = ds(vc0, dm(0.5, r1)); vy[k2] = ds(vc1, dm(0.5, r2)); vz[k2] = ds(vc2, dm(0.5, r3));
}

__device__ __forceinline__ void pair_execute_fp32(float* vx, float* vy, float* vz, float* ir, int k1, int k2,
                                                  const PairDraw& d, uint32_t w3, const DevConsts& C)
{
    const float v1x = vx[k1], v1y = vy[k1], v1z = vz[k1];
    const float v2x = vx[k2], v2y = vy[k2], v2z = vz[k2];
    const float vr0 = v1x - v2x, vr1 = v1y - v2y, vr2 = v1z - v2z;
    const float cr2 = vr0 * vr0 + vr1 * vr1 + vr2 * vr2;
    const float cr = psqrt(cr2);
    float preErt = 0.25f * cr2;
    const U4 b1 = d.block(1, C);
    const float uRel[2] = {unit32(w3), unit32(b1.x)};
    const float rChi = unit32(b1.y), th = unit32(b1.z);
    const float expLB = (float)C.expLB;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        float* irp = (h == 0) ? &ir[k1] : &ir[k2];
        if (uRel[h] <= C.prelaxF) {
            const float r = fminf(uRel[h] * C.invPrelaxF, 1.0f);
            const float preEr = *irp;
            const float postEr = (preErt + preEr) * (1.0f - exp2f(expLB * __log2f(r)));
            *irp = postEr;
            preErt = preErt + preEr - postEr;
        }
    }
    const float postVr = 2.0f * psqrt(preErt);
    const float vc0 = 0.5f * (v1x + v2x), vc1 = 0.5f * (v1y + v2y), vc2 = 0.5f * (v1z + v2z);
    const float cosChi =
        (C.alpha == 1.0) ? 2.0f * rChi - 1.0f : 2.0f * exp2f((float)C.invAlpha * __log2f(rChi)) - 1.0f;
    const float sinChi = psqrt(1.0f - cosChi * cosChi);
    // azimuth 2 pi th: sin and cos of 2 pi (th - 1/2) in [-pi, pi), negated
    const float ang = 6.283185307179586f * (th - 0.5f);
    const float sth = -__sinf(ang), cth = -__cosf(ang);
    const float vrp = psqrt(vr1 * vr1 + vr2 * vr2);
    const float scale = __fdividef(postVr, cr > 1.0e-30f ? cr : 1.0e-30f);
    const float vrpc = vrp > 1.0e-30f ? vrp : 1.0e-30f;
    float r1, r2, r3;
    if (vrp < 1e-6f) {
        r1 = scale * cosChi * vr0;
        r2 = scale * sinChi * vr0 * cth;
        r3 = scale * sinChi * vr0 * sth;
    } else {
        r1 = scale * (cosChi * vr0 + sinChi * sth * vrp);
        r2 = scale * (cosChi * vr1 + __fdividef(sinChi * (cr * vr2 * cth - vr0 * vr1 * sth), vrpc));
        r3 = scale * (cosChi * vr2 - __fdividef(sinChi * (cr * vr1 * cth + vr0 * vr2 * sth), vrpc));
    }
    vx[k1] = vc0 + 0.5f * r1; vy[k1] = vc1 + 0.5f * r2; vz[k1] = vc2 + 0.5f * r3;
    vx[k2] = vc0 - 0.5f * r1; vy[k2] = vc1 - 0.5f * r2; vz[k2] = vc2 - 0.5f * r3;
}

template <typename Real>
__device__ __forceinline__ void pair_execute(Real* vx, Real* vy, Real* vz, Real* ir, int stride, int k1, int k2,
                                             int c, int istep, int j, uint32_t w3, const DevConsts& C)
{
    PairDraw d;
    d.c = (uint32_t)c; d.istep = (uint32_t)istep; d.purpose = kPurposeCollide | ((uint32_t)j << 4);
    if constexpr (sizeof(Real) == 8) pair_execute_fp64(vx, vy, vz, ir, k1 * stride, k2 * stride, d, C);
    else pair_execute_fp32(vx, vy, vz, ir, k1 * stride, k2 * stride, d, w3, C);
}

// Candidate pair count of a cell from the majorant, with the carried
// remainder (collisionDSMC, src/ProcessDSMC.cpp:2631-2645), in the
// reference's evaluation order.
template <typename Real>
__device__ __forceinline__ int pair_count(const StepArgs<Real>& a, int c, int n, double& consCrm, double& crm0)
{
    crm0 = a.crmax[c];
    const double S = a.M.cellVolume[c];
    consCrm = collision_diameter(dm(crm0, a.C.vrms), a.C.cdPrefactor, a.C.eta);
    double t = dm(0.5, (double)n);
    t = dm(t, (double)(n - 1));
    t = dm(t, a.C.neff);
    t = dm(t, consCrm);
    t = dm(t, a.C.dtime);
    t = dm(t, a.C.dtref);
    const double pairs = da(dd(t, S), a.remColl[c]);
    const int npairs = (int)floor(pairs);
    a.remColl[c] = ds(pairs, (double)npairs);
    return npairs;
}

// The pair count and the majorant term of cell c as the classify pass
// computed them (pair_count), with the cell's crmax.
template <typename Real>
__device__ __forceinline__ int pair_fetch(const StepArgs<Real>& a, int c, double& consCrm, double& crm0)
{
    consCrm = a.cellCons[c];
    crm0 = a.crmax[c];
    return a.cellPairs[c];
}

// NTC collisions of one small cell by one thread: the candidate pairs one
// after another, particle k at v[k * stride].
template <typename Real>
__device__ void collide_cell_serial(Real* vx, Real* vy, Real* vz, Real* ir, int stride, int n, int c,
                                    const StepArgs<Real>& a, int istep, uint32_t& pairsOut, uint32_t& collOut)
{
    if (n <= 1) return;
    double consCrm, crm0;
    const int npairs = pair_fetch(a, c, consCrm, crm0);
    pairsOut += (uint32_t)npairs;
    if (!(consCrm > 0.0) || npairs <= 0) return;
    Real crmLocal = (Real)0;
    const Real crm0r = (Real)crm0;
    for (int j = 0; j < npairs; ++j) {
        int k1, k2;
        const PairDraw d = pair_draw(c, istep, j, n, a.C, k1, k2);
        if (pair_accept<Real>(vx, vy, vz, stride, k1, k2, d.b0.z, d.b0.w, a.C, consCrm, crm0r, crmLocal)) {
            pair_execute<Real>(vx, vy, vz, ir, stride, k1, k2, c, istep, j, d.b0.w, a.C);
            ++collOut;
        }
    }
    if ((double)crmLocal > crm0) a.crmax[c] = (double)crmLocal;
}

// NTC collisions of one cell by one warp (collisionDSMC,
// src/ProcessDSMC.cpp:2631-2665): the pair count from the majorant with the
// carried remainder, then candidate pairs j = 0, 1, ... each drawn from a
// Philox stream keyed by (cell, step, j).
//
// The pairs run as a sliding window: every lane holds one pending pair and
// claims both its particles with the pair index (atomicMin); a pair whose
// index is the lowest claim on both particles goes, and its lane takes the
// next unassigned pair. Pairs are handed out in increasing order, so a pair
// goes only after every lower pair that shares a particle with it, and the
// result equals running the pairs one after another. The lowest pending
// pair always goes, so the loop ends after at most npairs rounds.
// claim holds n ints (shared memory, or the output buffer's cell-id slots
// of the cell for large cells; the caller restores those).
template <typename Real>
__device__ void collide_cell(Real* vx, Real* vy, Real* vz, Real* ir, int* claim, int n, int c,
                             const StepArgs<Real>& a, int istep, uint32_t& pairsOut, uint32_t& collOut)
{
    const int lane = threadIdx.x & 31;
    if (n <= 1) return;
    double consCrm = 0.0, crm0 = 0.0;
    int npairs = 0;
    if (lane == 0) {
        npairs = pair_fetch(a, c, consCrm, crm0);
        pairsOut += (uint32_t)npairs;
    }
    npairs = __shfl_sync(kFull, npairs, 0);
    consCrm = __shfl_sync(kFull, consCrm, 0);
    crm0 = __shfl_sync(kFull, crm0, 0);
    if (!(consCrm > 0.0) || npairs <= 0) return;
    for (int k = lane; k < n; k += 32) claim[k] = INT_MAX;
    __syncwarp();
    Real crmLocal = (Real)0;
    const Real crm0r = (Real)crm0;
    const unsigned below = (1u << lane) - 1u;
    int next = 0;     // first pair not yet handed out (same in every lane)
    int j = -1;       // this lane's pending pair
    int k1 = 0, k2 = 0;
    PairDraw d;
    for (;;) {
        const unsigned idle = __ballot_sync(kFull, j < 0);
        if (j < 0) {
            const int jj = next + __popc(idle & below);
            if (jj < npairs) {
                j = jj;
                d = pair_draw(c, istep, j, n, a.C, k1, k2);
            }
        }
        next = min(npairs, next + __popc(idle));
        if (__ballot_sync(kFull, j >= 0) == 0u) break;
        if (j >= 0) {
            atomicMin(&claim[k1], j);
            atomicMin(&claim[k2], j);
        }
        __syncwarp();
        const bool go = j >= 0 && claim[k1] == j && claim[k2] == j;
        __syncwarp();
        if (go) {
            if (pair_accept<Real>(vx, vy, vz, 1, k1, k2, d.b0.z, d.b0.w, a.C, consCrm, crm0r, crmLocal)) {
                pair_execute<Real>(vx, vy, vz, ir, 1, k1, k2, c, istep, j, d.b0.w, a.C);
                ++collOut;
            }
            claim[k1] = INT_MAX;
            claim[k2] = INT_MAX;
            j = -1;
        }
        __syncwarp();
    }
    Real m = crmLocal;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const Real y = __shfl_xor_sync(kFull, m, o);
        m = y > m ? y : m;
    }
    if (lane == 0 && (double)m > crm0) a.crmax[c] = (double)m;
}

// The collision pass over the sorted buffer (collisionDSMC,
// src/ProcessDSMC.cpp:2621-2665). Cells are classified first
// (classify_kernel) and handed out dynamically, largest first:
// - huge cells (more than kArena particles): one at a time by a whole warp
//   (collide_cell), in place in the buffer;
// - large cells: two at a time per warp (collide_two_channels), staged in
//   shared memory;
// - small cells (at most kSmallMax particles): 32 at a time per warp, lane
//   l owning one cell and running its pairs alone, with the particles'
//   velocities and internal energies in shared memory at slot k * 32 + l
//   (lane l's slots sit in bank l, so the lanes never conflict).
// A cell's result depends on nothing but the cell, so neither the warp that
// takes it nor the order matters.
constexpr int kCellWarps = 2;
constexpr int kSmallMax = 16;
constexpr int kArena = 512;                   // staged particles per warp
constexpr int kSmallSlots = 32 * kSmallMax;
static_assert(kSmallSlots <= kArena, "small-cell slots must fit in the arena");

// per-warp shared memory: Real arena[4][kArena]; int claim[kArena]; int4 queue[64]
template <typename Real>
__host__ __device__ constexpr size_t warp_smem_bytes()
{
    return (size_t)kArena * (4 * sizeof(Real) + sizeof(int)) + 64 * sizeof(int4);
}
template <typename Real>
__host__ __device__ constexpr size_t cell_smem_bytes()
{
    return (size_t)kCellWarps * warp_smem_bytes<Real>();
}

// cellWork: [0] huge count, [1] large count, [2] small count,
//           [3] next huge/large item, [4] next small item
// cellList: huge cells from the front of [0, ncell), large cells from its
//           back, small cells from the front of [ncell, 2 ncell)
template <typename Real>
__global__ void classify_kernel(StepArgs<Real> a, int stageMax)
{
    const int lane = threadIdx.x & 31;
    const int* start = a.startA;
    const int ncell = a.M.ncell;
    int* list = a.cellList;
    int* work = a.cellWork;
    for (int base = blockIdx.x * blockDim.x; base < ncell; base += gridDim.x * blockDim.x) {
        const int c = base + threadIdx.x;
        const int s0 = c < ncell ? start[c] : 0;
        const int n = c < ncell ? start[c + 1] - s0 : -1;
        // the cell's candidate pair count, one thread per cell (the
        // collision kernels read it back with pair_fetch, or from the
        // cell's item record)
        int np = 0;
        double consCrm = 0.0, crm0 = 0.0;
        if (n > 1) {
            np = pair_count(a, c, n, consCrm, crm0);
            a.cellPairs[c] = np;
            a.cellCons[c] = consCrm;
        }
        const int cls = n < 0 ? -1 : (n > stageMax ? 0 : (n > kSmallMax ? 1 : 2));
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            const unsigned m = __ballot_sync(kFull, cls == k);
            if (!m) continue;
            const int leader = __ffs(m) - 1;
            int b = 0;
            if (lane == leader) b = atomicAdd(work + k, __popc(m));
            b = __shfl_sync(kFull, b, leader);
            if (cls == k) {
                const int pos = b + __popc(m & ((1u << lane) - 1u));
                if (k == 2) {
                    list[ncell + pos] = c;
                } else {
                    const int slot = k == 0 ? pos : ncell - 1 - pos;
                    list[slot] = c;
                    a.cellItem[slot] = make_int4(c, s0, n, np);
                    a.cellItemC[slot] = make_double2(consCrm, crm0);
                }
            }
        }
    }
}

// copy a cell's velocities and internal energies between the buffer (at s0)
// and v[comp][k * stride], whole warp. Into shared memory, the loads of up
// to 128 particles are issued before their stores (one round trip to
// memory for most cells instead of one per 32 particles).
template <typename Real, bool kToBuffer>
__device__ __forceinline__ void copy_cell(const PBuf<Real>& buf, int s0, int n, Real* const (&v)[4], int stride)
{
    const int lane = threadIdx.x & 31;
    Real* b[4] = {buf.v[0] + s0, buf.v[1] + s0, buf.v[2] + s0, buf.ir + s0};
    if constexpr (kToBuffer) {
        for (int k = lane; k < n; k += 32)
#pragma unroll
            for (int q = 0; q < 4; ++q) b[q][k] = v[q][k * stride];
    } else {
        for (int k0 = lane; k0 < n; k0 += 128) {
            Real t[4][4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + 32 * u;
#pragma unroll
                for (int q = 0; q < 4; ++q) t[u][q] = k < n ? b[q][k] : (Real)0;
            }
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = k0 + 32 * u;
                if (k < n)
#pragma unroll
                    for (int q = 0; q < 4; ++q) v[q][k * stride] = t[u][q];
            }
        }
    }
}

// Collisions of staged large cells, two cells per warp at a time, both in
// the warp's arena: channel 0's cell at slots [0, n0), channel 1's at
// [kArena - n1, kArena); a cell that does not fit beside the other channel's
// waits until that one is done. Each channel runs the sliding window of
// collide_cell (one pending pair per lane, claims by pair index); the pairs
// that go in a round are tested for acceptance by their own lanes, and the
// accepted ones, from both channels, are queued in shared memory and carried
// out by consecutive lanes, so the costly half of a collision runs once per
// round with most lanes busy. A channel whose pairs are done writes its
// cell back and takes the next. *item holds a cell item
// already taken from the list, or -1.
template <typename Real>
__device__ void collide_two_channels(const StepArgs<Real>& a, const PBuf<Real>& dst, const int* start, Real* arena,
                                     int* sclaim, int4* queue, int nItems, int nHuge, int istep, int item,
                                     uint32_t& pairs, uint32_t& colls)
{
    constexpr int N = kArena;
    const int lane = threadIdx.x & 31;
    const unsigned below = (1u << lane) - 1u;
    const int ncell = a.M.ncell;
    int cc[2] = {-1, -1}, cbase[2] = {0, 0}, cs0[2] = {0, 0}, cn[2] = {0, 0}, cnp[2] = {0, 0}, cnext[2] = {0, 0};
    double ccons[2] = {0.0, 0.0}, ccrm[2] = {0.0, 0.0};
    Real crmL[2] = {(Real)0, (Real)0};
    int sj[2] = {-1, -1}, sk1[2] = {0, 0}, sk2[2] = {0, 0};
    uint32_t sw2[2] = {0u, 0u}, sw3[2] = {0u, 0u};
    int held = item;      // an item taken but not yet placed
    bool more = true;
    // the next item index, taken one item ahead (lane 0): the atomic's
    // round trip overlaps the rounds of the cells in work. Indices are
    // handed out in increasing order and the loop runs until it sees one
    // past the end, so an index taken ahead is always used.
    int ahead = 0;
    if (lane == 0) ahead = atomicAdd(a.cellWork + 3, 1);
    for (;;) {
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            while (cc[ch] < 0 && (more || held >= 0)) {
                int it = held;
                if (it < 0) {
                    it = __shfl_sync(kFull, ahead, 0);
                    if (lane == 0 && it < nItems) ahead = atomicAdd(a.cellWork + 3, 1);
                }
                held = -1;
                if (it >= nItems) {
                    more = false;
                    break;
                }
                // the item's record (classify pass): one load instead of the
                // list, the starts and the pair count one after another
                const int slot = it < nHuge ? it : ncell - 1 - (it - nHuge);
                const int4 rec = a.cellItem[slot];
                const double2 rc = a.cellItemC[slot];
                const int c = rec.x, s0 = rec.y, n = rec.z;
                if (n > N) {   // never reached (huge items precede these): flag rather than overflow the arena
                    if (lane == 0) atomicOr(a.errorWord, kErrStageCell);
                    continue;
                }
                if (n > N - (cc[ch ^ 1] >= 0 ? cn[ch ^ 1] : 0)) {   // wait for the other channel
                    held = it;
                    break;
                }
                const int np = n > 1 ? rec.w : 0;
                const double consCrm = rc.x, crm0 = rc.y;
                if (lane == 0) pairs += (uint32_t)np;
                if (!(consCrm > 0.0) || np <= 0) continue;   // nothing changes: not staged
                const int base = ch == 0 ? 0 : N - n;
                Real* const v[4] = {arena + base, arena + N + base, arena + 2 * N + base, arena + 3 * N + base};
                copy_cell<Real, false>(dst, s0, n, v, 1);
                __syncwarp();
                for (int k = lane; k < n; k += 32) sclaim[base + k] = INT_MAX;
                __syncwarp();
                cc[ch] = c; cbase[ch] = base; cs0[ch] = s0; cn[ch] = n; cnp[ch] = np; cnext[ch] = 0;
                ccons[ch] = consCrm; ccrm[ch] = crm0; crmL[ch] = (Real)0;
            }
        }
        if (cc[0] < 0 && cc[1] < 0) break;
        // hand out the next pairs to idle lanes
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            if (cc[ch] < 0) continue;
            const unsigned idle = __ballot_sync(kFull, sj[ch] < 0);
            if (sj[ch] < 0) {
                const int jj = cnext[ch] + __popc(idle & below);
                if (jj < cnp[ch]) {
                    sj[ch] = jj;
                    int k1, k2;
                    const PairDraw d = pair_draw(cc[ch], istep, jj, cn[ch], a.C, k1, k2);
                    sk1[ch] = cbase[ch] + k1;
                    sk2[ch] = cbase[ch] + k2;
                    sw2[ch] = d.b0.z;
                    sw3[ch] = d.b0.w;
                }
            }
            cnext[ch] = min(cnp[ch], cnext[ch] + __popc(idle));
        }
        // claim both particles with the pair index; the lowest claim goes
#pragma unroll
        for (int ch = 0; ch < 2; ++ch)
            if (sj[ch] >= 0) {
                atomicMin(&sclaim[sk1[ch]], sj[ch]);
                atomicMin(&sclaim[sk2[ch]], sj[ch]);
            }
        __syncwarp();
        bool go[2], acc[2];
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) go[ch] = sj[ch] >= 0 && sclaim[sk1[ch]] == sj[ch] && sclaim[sk2[ch]] == sj[ch];
        __syncwarp();
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            acc[ch] = false;
            if (go[ch])
                acc[ch] = pair_accept<Real>(arena, arena + N, arena + 2 * N, 1, sk1[ch], sk2[ch], sw2[ch], sw3[ch], a.C,
                                            ccons[ch], (Real)ccrm[ch], crmL[ch]);
        }
        const unsigned m0 = __ballot_sync(kFull, acc[0]);
        const unsigned m1 = __ballot_sync(kFull, acc[1]);
        if (acc[0]) queue[__popc(m0 & below)] = make_int4(sk1[0] - cbase[0], sk2[0] - cbase[0], sj[0], (int)sw3[0]);
        if (acc[1])
            queue[__popc(m0) + __popc(m1 & below)] =
                make_int4(sk1[1] - cbase[1], sk2[1] - cbase[1], sj[1] | (1 << 30), (int)sw3[1]);
        __syncwarp();
        const int total = __popc(m0) + __popc(m1);
        for (int e = lane; e < total; e += 32) {
            const int4 q = queue[e];
            const int ch = q.z >> 30;
            const int base = ch ? cbase[1] : cbase[0];
            Real* b = arena + base;
            pair_execute<Real>(b, b + N, b + 2 * N, b + 3 * N, 1, q.x, q.y, ch ? cc[1] : cc[0], istep,
                               q.z & 0x3fffffff, (uint32_t)q.w, a.C);
        }
        if (lane == 0) colls += (uint32_t)total;
        __syncwarp();
#pragma unroll
        for (int ch = 0; ch < 2; ++ch)
            if (go[ch]) {
                sclaim[sk1[ch]] = INT_MAX;
                sclaim[sk2[ch]] = INT_MAX;
                sj[ch] = -1;
            }
        __syncwarp();
        // a channel whose pairs are all done finishes its cell
#pragma unroll
        for (int ch = 0; ch < 2; ++ch) {
            if (cc[ch] < 0) continue;
            if (__ballot_sync(kFull, sj[ch] >= 0) != 0u || cnext[ch] < cnp[ch]) continue;
            Real m = crmL[ch];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                const Real y = __shfl_xor_sync(kFull, m, o);
                m = y > m ? y : m;
            }
            if (lane == 0 && (double)m > ccrm[ch]) a.crmax[cc[ch]] = (double)m;
            const int base = cbase[ch];
            Real* const v[4] = {arena + base, arena + N + base, arena + 2 * N + base, arena + 3 * N + base};
            copy_cell<Real, true>(dst, cs0[ch], cn[ch], v, 1);
            __syncwarp();
            cc[ch] = -1;
        }
    }
}

// Nine resident blocks (18 warps) per SM: the arena (22.5 KB per block plus
// the 1 KB the runtime reserves) fits nine in 228 KB; the bound caps the
// registers to match (113 per thread).
template <typename Real>
__global__ void __launch_bounds__(kCellWarps * 32, 9) collide_kernel(StepArgs<Real> a)
{
    extern __shared__ __align__(16) unsigned char cellSmem[];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    unsigned char* wsm = cellSmem + (size_t)wib * warp_smem_bytes<Real>();
    Real* sv = reinterpret_cast<Real*>(wsm);
    int* sclaim = reinterpret_cast<int*>(wsm + (size_t)4 * kArena * sizeof(Real));
    int4* queue = reinterpret_cast<int4*>(wsm + (size_t)kArena * (4 * sizeof(Real) + sizeof(int)));
    Real* const stage[4] = {sv, sv + kSmallSlots, sv + 2 * kSmallSlots, sv + 3 * kSmallSlots};
    const int istep = a.ctl->istep;
    const PBuf<Real> buf = a.A;
    const int* start = a.startA;
    const int ncell = a.M.ncell;
    const int nHuge = a.cellWork[0], nLarge = a.cellWork[1], nSmall = a.cellWork[2];
    uint32_t pairs = 0, colls = 0, big = 0;

    // ---- huge cells, one at a time by the whole warp, in place
    int item = -1;
    for (;;) {
        int it = 0;
        if (lane == 0) it = atomicAdd(a.cellWork + 3, 1);
        it = __shfl_sync(kFull, it, 0);
        if (it >= nHuge + nLarge) break;
        if (it >= nHuge) {   // a large cell: the two-channel loop takes it
            item = it;
            break;
        }
        const int c = a.cellList[it];
        const int s0 = start[c];
        const int n = start[c + 1] - s0;
        if (lane == 0) ++big;
        collide_cell<Real>(buf.v[0] + s0, buf.v[1] + s0, buf.v[2] + s0, buf.ir + s0, buf.cell + s0, n, c, a, istep,
                           pairs, colls);
        __syncwarp();
        for (int k = lane; k < n; k += 32) buf.cell[s0 + k] = c;   // the claims used the cell ids
        __syncwarp();
    }

    // ---- large cells, two at a time
    if (item >= 0)
        collide_two_channels<Real>(a, buf, start, sv, sclaim, queue, nHuge + nLarge, nHuge, istep, item, pairs, colls);

    // ---- small cells, 32 per warp, one lane each
    for (;;) {
        int g = 0;
        if (lane == 0) g = atomicAdd(a.cellWork + 4, 32);
        g = __shfl_sync(kFull, g, 0);
        if (g >= nSmall) break;
        const bool mine = g + lane < nSmall;
        const int myc = mine ? a.cellList[ncell + g + lane] : 0;
        const int ms0 = mine ? start[myc] : 0;
        const int mn = mine ? start[myc + 1] - ms0 : 0;
        const unsigned mask = __ballot_sync(kFull, mine && mn > 1);
        for (unsigned m = mask; m; m &= m - 1) {
            const int l = __ffs(m) - 1;
            Real* const to[4] = {stage[0] + l, stage[1] + l, stage[2] + l, stage[3] + l};
            copy_cell<Real, false>(buf, __shfl_sync(kFull, ms0, l), __shfl_sync(kFull, mn, l), to, 32);
        }
        __syncwarp();
        if ((mask >> lane) & 1u)
            collide_cell_serial<Real>(stage[0] + lane, stage[1] + lane, stage[2] + lane, stage[3] + lane, 32, mn, myc,
                                      a, istep, pairs, colls);
        __syncwarp();
        for (unsigned m = mask; m; m &= m - 1) {
            const int l = __ffs(m) - 1;
            Real* const from[4] = {stage[0] + l, stage[1] + l, stage[2] + l, stage[3] + l};
            copy_cell<Real, true>(buf, __shfl_sync(kFull, ms0, l), __shfl_sync(kFull, mn, l), from, 32);
        }
        __syncwarp();
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        pairs += __shfl_xor_sync(kFull, pairs, o);
        colls += __shfl_xor_sync(kFull, colls, o);
        big += __shfl_xor_sync(kFull, big, o);
    }
    if (lane == 0) {
        if (pairs) atomicAdd(a.counters + C_PAIRS, (unsigned long long)pairs);
        if (colls) atomicAdd(a.counters + C_COLLISIONS, (unsigned long long)colls);
        if (big) atomicAdd(a.counters + C_BIG_CELLS, (unsigned long long)big);
    }
}

// resident blocks per SM of each cell-kernel variant, set by prepare_kernels
template <typename Real>
struct CellOcc {
    static int blocks;
};
template <typename Real>
int CellOcc<Real>::blocks = 1;

template <typename Real>
cudaError_t prepare_kernels()
{
    cudaError_t e = cudaFuncSetAttribute(collide_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)cell_smem_bytes<Real>());
    if (e != cudaSuccess) return e;
    int nb = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, collide_kernel<Real>, kCellWarps * 32,
                                                      cell_smem_bytes<Real>());
    if (e != cudaSuccess) return e;
    CellOcc<Real>::blocks = nb > 0 ? nb : 1;
    const void* stay[3] = {(const void*)move_stay_kernel<Real, 1>, (const void*)move_stay_kernel<Real, 2>,
                           (const void*)move_stay_kernel<Real, 4>};
    for (int k = 0; k < 3; ++k) {
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, stay[k], 256, 0);
        if (e != cudaSuccess) return e;
        StayOcc<Real>::blocks[k] = nb > 0 ? nb : 1;
    }
    return cudaSuccess;
}

template <typename Real>
void launch_collide(const StepArgs<Real>& a, const LaunchShape& L, cudaStream_t s)
{
    const int ncell = a.M.ncell;
    cudaMemsetAsync(a.cellWork, 0, 8 * sizeof(int), s);
    int gc = (ncell + 255) / 256;
    if (gc > L.smCount * 8) gc = L.smCount * 8;
    classify_kernel<Real><<<gc > 0 ? gc : 1, 256, 0, s>>>(a, kArena);
    int g = (ncell + kCellWarps - 1) / kCellWarps;
    const int cap = L.smCount * min(CellOcc<Real>::blocks, max(1, L.collideBlocksPerSm));
    if (g > cap) g = cap;
    collide_kernel<Real><<<g > 0 ? g : 1, kCellWarps * 32, cell_smem_bytes<Real>(), s>>>(a);
}

// ===========================================================================
// sampling
// ===========================================================================

// Raw moments of one cell's particles, summed in particle order with each
// operation rounded on its own (the oracle's order and rounding).
template <typename Real>
__device__ __forceinline__ void cell_moments(const PBuf<Real>& b, int s0, int n, double m[18])
{
#pragma unroll
    for (int k = 0; k < 18; ++k) m[k] = 0.0;
    for (int k = s0; k < s0 + n; ++k) {
        const double x = (double)b.v[0][k], y = (double)b.v[1][k], z = (double)b.v[2][k], I = (double)b.ir[k];
        const double v2 = da(da(dm(x, x), dm(y, y)), dm(z, z));
        m[0] = da(m[0], 1.0); m[1] = da(m[1], x); m[2] = da(m[2], y); m[3] = da(m[3], z); m[4] = da(m[4], v2);
        m[5] = da(m[5], dm(x, x)); m[6] = da(m[6], dm(x, y)); m[7] = da(m[7], dm(y, y));
        m[8] = da(m[8], dm(y, z)); m[9] = da(m[9], dm(z, z)); m[10] = da(m[10], dm(z, x));
        m[11] = da(m[11], dm(x, v2)); m[12] = da(m[12], dm(y, v2)); m[13] = da(m[13], dm(z, v2));
        m[14] = da(m[14], I); m[15] = da(m[15], dm(x, I)); m[16] = da(m[16], dm(y, I)); m[17] = da(m[17], dm(z, I));
    }
}

// updateStepWindowMoments, :3106-3113, for moment k of a cell: the
// exponential window (local), the steady sum past NSS (final_record) and the
// GSIS window sum (every NEVERY steps)
// (s, sSteady, sWindow: the three accumulators' values before the step).
template <typename Real>
__device__ __forceinline__ void fold_moment(const StepArgs<Real>& a, double* acc, int k, double v, int istep,
                                            double s, double sSteady, double sWindow)
{
    const bool every = (istep % a.C.nevery) == 0;
    const double na = (double)a.C.nscheme;
    const double w = (istep <= a.C.nscheme) ? 1.0 : dd(ds(na, 1.0), na);
    const bool steady = istep > a.C.nss;
    acc[k] = (w == 1.0) ? da(s, v) : da(dm(w, s), v);
    if (steady) acc[18 + k] = da(sSteady, v);
    if (every) acc[36 + k] = da(sWindow, v);
}

// The rest of statistic_macro for cell c once its moments are folded in:
// the sparse-cell state machine and, at an exchange step, the record fields
// from the GSIS window.
template <typename Real>
__device__ __forceinline__ void sample_cell_tail(const StepArgs<Real>& a, int c, double* acc, int istep)
{
    const double S = a.M.cellVolume[c];
    const bool every = (istep % a.C.nevery) == 0;
    const int ngsis = a.C.nevery * a.C.nrepeat;
    unsigned char st = a.sparseState[c];
    int accum = a.sparseAccum[c];
    if (every && (st == 1 || st == 2)) {
        if (accum < 0) accum = 0;
        ++accum;
    }
    if (ngsis > 0 && istep % ngsis == 0) {
        const double* inter = acc + 36;
        const double ws = inter[0];
        const bool finite = isfinite(ws);
        bool sparse = (st == 1 || st == 2);
        if (!sparse && finite && ws < 3.0) {
            st = 1;
            accum = a.C.nrepeat > 1 ? a.C.nrepeat : 1;
            sparse = true;
        }
        const bool valid = (ws >= 3.0) && finite;
        a.windowSamples[c] = ws;
        a.windowValid[c] = valid ? 1 : 0;
        double out[18];
        if (sparse) {
            averaged_macro(inter, (double)(accum > 1 ? accum : 1), S, a.C.neff, a.C.nref, a.C.dr, out);
            for (int k = 0; k < 18; ++k) a.record[(size_t)c * 18 + k] = out[k];
        } else if (valid) {
            averaged_macro(inter, (double)a.C.nrepeat, S, a.C.neff, a.C.nref, a.C.dr, out);
            for (int k = 0; k < 18; ++k) a.record[(size_t)c * 18 + k] = out[k];
        }
        if (!sparse)
            for (int k = 0; k < 18; ++k) acc[36 + k] = 0.0;
    }
    a.sparseState[c] = st;
    a.sparseAccum[c] = accum;
}

// Fold one step's moments of cell c into its accumulators, by one thread:
// statistic_macro, src/ProcessDSMC.cpp:2784-2859 (statistic_macroPre,
// :3312-3326, when pre).
template <typename Real>
__device__ __forceinline__ void sample_cell(const StepArgs<Real>& a, int c, const double* mom, int istep, bool pre)
{
    const double S = a.M.cellVolume[c];
    if (a.stepMom)
        for (int k = 0; k < 18; ++k) a.stepMom[(size_t)c * 18 + k] = mom[k];
    if (pre) {
        double out[18];
        local_macro_pre(mom, S, a.C.neff, a.C.nref, a.C.dr, out);
        for (int k = 0; k < 18; ++k) a.local[(size_t)c * 18 + k] = out[k];
        record_macro_pre(mom, S, a.C.neff, a.C.nref, a.C.dr, out);
        for (int k = 0; k < 18; ++k) a.record[(size_t)c * 18 + k] = out[k];
        return;
    }
    double* acc = a.acc + (size_t)c * 54;
    for (int k = 0; k < 18; ++k) fold_moment(a, acc, k, mom[k], istep, acc[k], acc[18 + k], acc[36 + k]);
    sample_cell_tail(a, c, acc, istep);
}


// statistic_macro / statistic_macroPre over the sorted buffer: one thread
// per cell.
template <typename Real>
__global__ void __launch_bounds__(128) sample_kernel(StepArgs<Real> a, int pre)
{
    const int istep = a.ctl->istep;
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < a.M.ncell; c += gridDim.x * blockDim.x) {
        const int s0 = a.startA[c];
        double mom[18];
        cell_moments<Real>(a.A, s0, a.startA[c + 1] - s0, mom);
        sample_cell<Real>(a, c, mom, istep, pre != 0);
    }
}

// statistic_macro of the mixed path, one warp per cell: the lanes sum the
// cell's particles 32 apart (coalesced loads), lane q < 18 then adds up
// moment q of the 32 lanes (four groups of eight, through shared memory)
// and folds it into the cell's accumulators, and lane 0 runs the rest. Its
// FP64 sums run in another order than the one-thread sums, which the FP64
// path keeps (they are the reference's order).
constexpr int kSampleWarps = 8;

__global__ void __launch_bounds__(kSampleWarps * 32, 3) sample_warp_kernel(StepArgs<float> a)
{
    __shared__ double part[kSampleWarps][18][33];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int istep = a.ctl->istep;
    double (*mine)[33] = part[wib];
    for (int c = blockIdx.x * kSampleWarps + wib; c < a.M.ncell; c += gridDim.x * kSampleWarps) {
        const int s0 = a.startA[c];
        const int e = a.startA[c + 1];
        double* acc = a.acc + (size_t)c * 54;
        // the accumulators' old values, loaded while the particles are summed
        double o0 = 0.0, o1 = 0.0, o2 = 0.0;
        if (lane < 18) {
            o0 = acc[lane]; o1 = acc[18 + lane]; o2 = acc[36 + lane];
        }
        double m[18];
#pragma unroll
        for (int q = 0; q < 18; ++q) m[q] = 0.0;
        auto add = [&](float fx, float fy, float fz, float fi) {
            const double x = (double)fx, y = (double)fy, z = (double)fz, I = (double)fi;
            const double v2 = da(da(dm(x, x), dm(y, y)), dm(z, z));
            m[0] = da(m[0], 1.0); m[1] = da(m[1], x); m[2] = da(m[2], y); m[3] = da(m[3], z); m[4] = da(m[4], v2);
            m[5] = da(m[5], dm(x, x)); m[6] = da(m[6], dm(x, y)); m[7] = da(m[7], dm(y, y));
            m[8] = da(m[8], dm(y, z)); m[9] = da(m[9], dm(z, z)); m[10] = da(m[10], dm(z, x));
            m[11] = da(m[11], dm(x, v2)); m[12] = da(m[12], dm(y, v2)); m[13] = da(m[13], dm(z, v2));
            m[14] = da(m[14], I); m[15] = da(m[15], dm(x, I)); m[16] = da(m[16], dm(y, I)); m[17] = da(m[17], dm(z, I));
        };
        // two particles per lane and iteration, their loads issued first
        int k = s0 + lane;
        for (; k + 32 < e; k += 64) {
            const float x1 = a.A.v[0][k], y1 = a.A.v[1][k], z1 = a.A.v[2][k], i1 = a.A.ir[k];
            const float x2 = a.A.v[0][k + 32], y2 = a.A.v[1][k + 32], z2 = a.A.v[2][k + 32], i2 = a.A.ir[k + 32];
            add(x1, y1, z1, i1);
            add(x2, y2, z2, i2);
        }
        if (k < e) add(a.A.v[0][k], a.A.v[1][k], a.A.v[2][k], a.A.ir[k]);
#pragma unroll
        for (int q = 0; q < 18; ++q) mine[q][lane] = m[q];
        __syncwarp();
        double mq = 0.0;
        if (lane < 18) {
            // four partial sums of eight lanes each, then their pairs
            double t[4];
#pragma unroll
            for (int g = 0; g < 4; ++g) {
                t[g] = mine[lane][8 * g];
#pragma unroll
                for (int l = 1; l < 8; ++l) t[g] = da(t[g], mine[lane][8 * g + l]);
            }
            mq = da(da(t[0], t[1]), da(t[2], t[3]));
        }
        __syncwarp();   // the rows are reused for the next cell
        if (lane < 18) {
            if (a.stepMom) a.stepMom[(size_t)c * 18 + lane] = mq;
            fold_moment(a, acc, lane, mq, istep, o0, o1, o2);
        }
        __syncwarp();   // lane 0 reads the folded window sums
        if (lane == 0) sample_cell_tail(a, c, acc, istep);
    }
}

template <typename Real>
void launch_sample(const StepArgs<Real>& a, bool pre, const LaunchShape& L, cudaStream_t s)
{
    if constexpr (sizeof(Real) == 4) {
        if (!pre) {
            int g = (a.M.ncell + kSampleWarps - 1) / kSampleWarps;
            if (g > L.smCount * 32) g = L.smCount * 32;
            sample_warp_kernel<<<g > 0 ? g : 1, kSampleWarps * 32, 0, s>>>(a);
            return;
        }
    }
    int g = (a.M.ncell + 127) / 128;
    if (g > L.smCount * 16) g = L.smCount * 16;
    sample_kernel<Real><<<g > 0 ? g : 1, 128, 0, s>>>(a, pre ? 1 : 0);
}

// ===========================================================================
// initial fill (Np_tri_inititial / meshfillpar / velocityLocationGenerate,
// src/MeshparticalInitial.cpp:481-721): particles already counted per cell
// (startA) and per placement tetrahedron (tetFirst: the cell-local index of
// each tetrahedron's first particle, counted on the host) take, in
// tetrahedron order, a point of their tetrahedron from the reference's
// normalised-uniform weights and a velocity u + sig * (unit Box-Muller
// triple: sqrt(-2 ln r) sin th, sqrt(-2 ln r) cos th, sqrt(-2 ln r2) sin th2)
// with Ir = -ln(r3) tN / 2; u = 0, sig = 1, tN = 1 is the reference's own
// unit Maxwellian at rest. Particle k of cell c draws from the Philox
// counters (c, k, kPurposeFill, 0..4): (r, th), (r2, th2), (r3, w0),
// (w1, w2), (w3, -).
// ===========================================================================
template <typename Real>
__global__ void __launch_bounds__(256) fill_kernel(StepArgs<Real> a, FillParams f, const int* __restrict__ tetFirst)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    constexpr bool mixed = sizeof(Real) == 4;
    constexpr double kTwoPi = 6.283185307179586;   // 2 * M_PI
    for (int c = warp; c < a.M.ncell; c += nwarps) {
        const int s0 = a.startA[c];
        const int n = a.startA[c + 1] - s0;
        const int t0 = a.M.placeOff[c], t1 = a.M.placeOff[c + 1];
        if (n == 0 || t1 <= t0) continue;
        const double cx = a.M.cellCenter[(size_t)c * 3 + 0], cy = a.M.cellCenter[(size_t)c * 3 + 1],
                     cz = a.M.cellCenter[(size_t)c * 3 + 2];
        for (int k = lane; k < n; k += 32) {
            int t = t0;
            for (int q = t0 + 1; q < t1; ++q)
                if (tetFirst[q] <= k) t = q;
            const uint32_t cc = (uint32_t)c, kk = (uint32_t)k;
            const U4 b0 = philox4x32_10(U4{cc, kk, kPurposeFill, 0u}, f.keyLo, f.keyHi);
            const U4 b1 = philox4x32_10(U4{cc, kk, kPurposeFill, 1u}, f.keyLo, f.keyHi);
            const U4 b2 = philox4x32_10(U4{cc, kk, kPurposeFill, 2u}, f.keyLo, f.keyHi);
            const U4 b3 = philox4x32_10(U4{cc, kk, kPurposeFill, 3u}, f.keyLo, f.keyHi);
            const U4 b4 = philox4x32_10(U4{cc, kk, kPurposeFill, 4u}, f.keyLo, f.keyHi);
            const double rad1 = sqrt(dm(-2.0, log(unit64(b0.x, b0.y))));
            const double th1 = dm(kTwoPi, unit64(b0.z, b0.w));
            const double rad2 = sqrt(dm(-2.0, log(unit64(b1.x, b1.y))));
            const double th2 = dm(kTwoPi, unit64(b1.z, b1.w));
            const double ir = dm(dm(-log(unit64(b2.x, b2.y)), f.tN), 0.5);
            double x[3];
            place_point(a.M.placeV + (size_t)t * 12, unit64(b2.z, b2.w), unit64(b3.x, b3.y), unit64(b3.z, b3.w),
                        unit64(b4.x, b4.y), x);
            const int o = s0 + k;
            if constexpr (mixed) {
                a.A.x[0][o] = (Real)(x[0] - cx); a.A.x[1][o] = (Real)(x[1] - cy); a.A.x[2][o] = (Real)(x[2] - cz);
            } else {
                a.A.x[0][o] = x[0]; a.A.x[1][o] = x[1]; a.A.x[2][o] = x[2];
            }
            a.A.v[0][o] = (Real)da(f.u[0], dm(f.sig, dm(rad1, sin(th1))));
            a.A.v[1][o] = (Real)da(f.u[1], dm(f.sig, dm(rad1, cos(th1))));
            a.A.v[2][o] = (Real)da(f.u[2], dm(f.sig, dm(rad2, sin(th2))));
            a.A.ir[o] = (Real)ir;
            a.A.cell[o] = c;
        }
    }
}

template <typename Real>
void launch_fill(const StepArgs<Real>& a, const FillParams& f, const int* tetFirst, const LaunchShape& L,
                 cudaStream_t s)
{
    fill_kernel<Real><<<L.smCount * 8, 256, 0, s>>>(a, f, tetFirst);
}

void launch_scan_counts(const int* countSlot, int ncell, int* partial, int* start, StepCtl* ctl, cudaStream_t s)
{
    scan_partial_kernel<<<kScanBlocks, 256, 0, s>>>(countSlot, ncell, partial);
    scan_final_kernel<<<kScanBlocks, 256, 0, s>>>(countSlot, ncell, partial, start, ctl);
}

// ===========================================================================
// macro fields on demand (local from the exponential window, final_record
// from the steady sum): writeAveragedMacro, src/ProcessDSMC.cpp:2790-2820
// ===========================================================================
__global__ void macro_kernel(DevMesh M, DevConsts C, const double* acc, int set, double count, double* out)
{
    for (int c = blockIdx.x * blockDim.x + threadIdx.x; c < M.ncell; c += gridDim.x * blockDim.x) {
        double m[18];
        for (int k = 0; k < 18; ++k) m[k] = acc[(size_t)c * 54 + set * 18 + k];
        double o[18];
        averaged_macro(m, count, M.cellVolume[c], C.neff, C.nref, C.dr, o);
        for (int k = 0; k < 18; ++k) out[(size_t)c * 18 + k] = o[k];
    }
}

void launch_macro(const DevMesh& M, const DevConsts& C, const double* acc, int set, double count, double* out,
                  int ncell, cudaStream_t s)
{
    int g = (ncell + 255) / 256;
    if (g > 2048) g = 2048;
    macro_kernel<<<g > 0 ? g : 1, 256, 0, s>>>(M, C, acc, set, count, out);
}

// ===========================================================================
// particle upload from cell-major host arrays
// ===========================================================================
__global__ void upload_check_kernel(const int* __restrict__ cell, int n, int ncell, int* flags, int* start)
{
    int bad = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const int c = cell[i];
        const int prev = i > 0 ? cell[i - 1] : -1;
        if (c < 0 || c >= ncell) { bad |= 1; continue; }
        if (prev > c) { bad |= 2; continue; }
        // cells prev+1 .. c begin at slot i (in range and ordered here; the
        // host uses start only when no thread flagged anything)
        const int lo = prev < 0 ? 0 : prev + 1;
        for (int q = lo; q <= c; ++q) start[q] = i;
        if (i == n - 1)
            for (int q = c + 1; q <= ncell; ++q) start[q] = n;
    }
    if (bad) atomicOr(flags, bad);
}

void launch_upload_check(const int* cell, int n, int ncell, int* flags, int* start, cudaStream_t s)
{
    int g = (n + 255) / 256;
    g = g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g);
    upload_check_kernel<<<g, 256, 0, s>>>(cell, n, ncell, flags, start);
}

__global__ void upload_convert_kernel(const double* __restrict__ in, const int* __restrict__ cell,
                                      const double* __restrict__ center, int comp, float* __restrict__ out, int n)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double v = in[i];
        if (comp < 3) v = v - center[(size_t)cell[i] * 3 + comp];
        out[i] = (float)v;
    }
}

void launch_upload_convert(const double* in, const int* cell, const double* center, int comp, float* out, int n,
                           cudaStream_t s)
{
    int g = (n + 255) / 256;
    g = g < 1 ? 1 : (g > 148 * 16 ? 148 * 16 : g);
    upload_convert_kernel<<<g, 256, 0, s>>>(in, cell, center, comp, out, n);
}

// ===========================================================================
// tracing check (dsmc_trace)
// ===========================================================================
template <typename Real>
__global__ void trace_check_kernel(DevMesh M, DevConsts C, int n, const Real* px, const Real* py, const Real* pz,
                                   const Real* vx, const Real* vy, const Real* vz, const double* dt,
                                   const int* cell, int stopAtWall, int* oCell, int* oIfout, int* oFace,
                                   int* oTri, int* oNcross, int* oLast, Real* ox, Real* oy, Real* oz, Real* ovx,
                                   Real* ovy, Real* ovz, double* odt, unsigned long long* counters)
{
    TraceCounts cnt{};
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        PRegs<Real> p;
        int c = cell[i];
        if constexpr (sizeof(Real) == 8) {
            p.x[0] = px[i]; p.x[1] = py[i]; p.x[2] = pz[i];
        } else {
            const double* cc = M.cellCenter + (size_t)c * 3;
            p.x[0] = da(cc[0], (double)px[i]); p.x[1] = da(cc[1], (double)py[i]); p.x[2] = da(cc[2], (double)pz[i]);
        }
        p.v[0] = vx[i]; p.v[1] = vy[i]; p.v[2] = vz[i];
        p.ir = (Real)0;
        Stream rs;
        rs.init((uint32_t)i, 0u, kPurposeWall, C.seedLo, C.seedHi);
        double dtleft = dt[i];
        TraceLog log{-1, 0, 0};
        const int out = trace_particle<Real>(M, C, p, c, -1, -1, dtleft, rs, 0, nullptr, cnt, stopAtWall != 0, &log);
        oCell[i] = (out == kTraceRemoved) ? -1 : c;
        oIfout[i] = (out >= 0) ? out : -1;
        oFace[i] = log.hitFace;
        oTri[i] = log.hitTri;
        oNcross[i] = log.ncross;
        if constexpr (sizeof(Real) == 8) {
            ox[i] = p.x[0]; oy[i] = p.x[1]; oz[i] = p.x[2];
        } else {
            // relative to the centre of the last cell the particle was in
            const double* cc = M.cellCenter + (size_t)c * 3;
            ox[i] = (float)ds(p.x[0], cc[0]); oy[i] = (float)ds(p.x[1], cc[1]); oz[i] = (float)ds(p.x[2], cc[2]);
        }
        ovx[i] = p.v[0]; ovy[i] = p.v[1]; ovz[i] = p.v[2];
        odt[i] = dtleft;
        oLast[i] = c;   // cell the position is relative to (mixed precision)
    }
    flush_counts(counters, cnt);
}

template <typename Real>
void launch_trace_check(const DevMesh& M, const DevConsts& C, int n, const Real* px, const Real* py, const Real* pz,
                        const Real* vx, const Real* vy, const Real* vz, const double* dt, const int* cell,
                        int stopAtWall, int* oCell, int* oIfout, int* oFace, int* oTri, int* oNcross, int* oLast,
                        Real* ox, Real* oy, Real* oz, Real* ovx, Real* ovy, Real* ovz, double* odt,
                        unsigned long long* counters, cudaStream_t s)
{
    int g = (n + 255) / 256;
    if (g > 4096) g = 4096;
    trace_check_kernel<Real><<<g > 0 ? g : 1, 256, 0, s>>>(M, C, n, px, py, pz, vx, vy, vz, dt, cell, stopAtWall,
                                                           oCell, oIfout, oFace, oTri, oNcross, oLast, ox, oy, oz,
                                                           ovx, ovy, ovz, odt, counters);
}

#define DSMC_INSTANTIATE(Real)                                                                                   \
    template void launch_inject<Real>(const StepArgs<Real>&, const LaunchShape&, cudaStream_t);                  \
    template void launch_move<Real>(const StepArgs<Real>&, const LaunchShape&, cudaStream_t);                    \
    template void launch_sort<Real>(const StepArgs<Real>&, const LaunchShape&, cudaStream_t);                    \
    template void launch_collide<Real>(const StepArgs<Real>&, const LaunchShape&, cudaStream_t);                 \
    template void launch_sample<Real>(const StepArgs<Real>&, bool, const LaunchShape&, cudaStream_t);            \
    template void launch_fill<Real>(const StepArgs<Real>&, const FillParams&, const int*, const LaunchShape&,    \
                                    cudaStream_t);                                                               \
    template cudaError_t prepare_kernels<Real>();                                                                \
    template void launch_trace_check<Real>(const DevMesh&, const DevConsts&, int, const Real*, const Real*,       \
                                           const Real*, const Real*, const Real*, const Real*, const double*,    \
                                           const int*, int, int*, int*, int*, int*, int*, int*, Real*, Real*,    \
                                           Real*, Real*, Real*, Real*, double*, unsigned long long*, cudaStream_t);
DSMC_INSTANTIATE(float)
DSMC_INSTANTIATE(double)

}  // namespace dsmc
