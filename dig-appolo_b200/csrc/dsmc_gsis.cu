// GSIS particle update on the device: ProcessGSIS::molecular_velocity_change
// with replication, deletion, MaxwellianSample and randomlocation
// (src/ProcessGSIS.cpp:2239-2530), between two steps.
//
// For every cell before the first one whose NS density or velocity is NaN,
// and not skipped by the acceptance gate, the particle count is brought to
// the NS count Iround(rho_ns V n_ref / Neff) by copying uniformly chosen
// particles of the growing bucket to new random points of the cell (or, in
// an empty cell, sampling a Maxwellian at the NS state) or by deleting
// uniformly chosen particles (the last one fills the hole), and then every
// particle of the cell is mapped v -> k v + b, Ir -> kr Ir so that the cell's
// mean velocity, temperature and rotational temperature equal the NS values.
//
// Device layout: the cell-sorted buffer A becomes the cell-sorted buffer B.
// A count pass writes each cell's new count into its countSlot row and the
// sort's scan lays out B; a warp per cell then writes the cell's particles
// into B in the reference's bucket order (the survivors of the swap-and-pop
// deletions, or the old particles followed by the copies in push order) and
// applies the linear map, the sums taken in bucket order as the reference
// takes them. Random choices come from Philox counters keyed by cell and
// draw index, so results do not depend on the launch shape.
#include "dsmc_kernels.cuh"

namespace dsmc {

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr double kTwoPi = 6.283185307179586;   // 2 * M_PI

__device__ __forceinline__ U4 gsis_draw(const GsisArgs& g, int c, int j, uint32_t sub, uint32_t block)
{
    return philox4x32_10(U4{(uint32_t)c, (uint32_t)j, g.purpose | (sub << 4), block}, g.keyLo, g.keyHi);
}

// uniform_int_distribution(0, m - 1) from a uniform in (0, 1)
__device__ __forceinline__ int pick_index(double u, int m)
{
    int k = (int)dm(u, (double)m);
    return k > m - 1 ? m - 1 : k;
}

__device__ __forceinline__ void warp_tally(unsigned long long* t, unsigned long long a, unsigned long long b,
                                           unsigned long long c, unsigned long long d)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(kFull, a, o);
        b += __shfl_xor_sync(kFull, b, o);
        c += __shfl_xor_sync(kFull, c, o);
        d += __shfl_xor_sync(kFull, d, o);
    }
    if ((threadIdx.x & 31) == 0) {
        if (a) atomicAdd(t + 0, a);
        if (b) atomicAdd(t + 1, b);
        if (c) atomicAdd(t + 2, c);
        if (d) atomicAdd(t + 3, d);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// target counts (molecular_velocity_change, src/ProcessGSIS.cpp:2255-2289)
// ---------------------------------------------------------------------------
template <typename Real>
__global__ void __launch_bounds__(256) gsis_count_kernel(StepArgs<Real> a, GsisArgs g)
{
    unsigned long long updated = 0, skipped = 0, added = 0, removed = 0;
    const int ncell = a.M.ncell;
    const int stride = gridDim.x * blockDim.x;
    const int first = blockIdx.x * blockDim.x + threadIdx.x;
    // whole warps loop together (the tally is a warp reduction)
    const int rounds = (ncell + stride - 1) / stride;
    for (int r = 0; r < rounds; ++r) {
        const int c = first + r * stride;
        if (c < ncell) {
            const int n0 = a.startA[c + 1] - a.startA[c];
            int target = n0, flag = 0;
            if (c < g.firstNan) {
                if (g.accepted && g.accepted[c] == 0) {
                    ++skipped;
                } else {
                    flag = 1;
                    ++updated;
                    const double* ns = g.ns + (size_t)c * 6;
                    // n_ns = nsresult * (area * n_ref) / Neff, then Iround
                    // (src/MeshparticalInitial.cpp:730-742)
                    const double x = __ddiv_rn(dm(ns[0], dm(a.M.cellVolume[c], a.C.nref)), a.C.neff);
                    const double fl = floor(x);
                    const U4 b = gsis_draw(g, c, 0, 0u, 0u);
                    const double nns = (unit64(b.x, b.y) < ds(x, fl)) ? da(fl, 1.0) : fl;
                    if (nns > (double)n0) {
                        if (!(nns < 1073741824.0)) {
                            atomicOr(a.errorWord, kErrGsisCount);
                        } else if (!(n0 == 0 && ns[4] < 0.0)) {
                            // replication refuses an empty cell with T_ns < 0
                            target = (int)nns;
                        }
                    } else if (nns < (double)n0) {
                        // deletion refuses to remove more than the cell holds
                        if (nns >= 0.0) target = (int)nns;
                    }
                }
            }
            int* row = a.countSlot + (size_t)c * kSlots;
            *reinterpret_cast<int4*>(row) = make_int4(target, 0, 0, 0);
            *reinterpret_cast<int4*>(row + 4) = make_int4(0, 0, 0, 0);
            g.flag[c] = flag;
            if (target > n0) added += (unsigned long long)(target - n0);
            else removed += (unsigned long long)(n0 - target);
        }
        warp_tally(g.tally, updated, skipped, added, removed);
        updated = skipped = added = removed = 0;
    }
}

template <typename Real>
void launch_gsis_count(const StepArgs<Real>& a, const GsisArgs& g, cudaStream_t s)
{
    int blocks = (a.M.ncell + 255) / 256;
    if (blocks > 4096) blocks = 4096;
    gsis_count_kernel<Real><<<blocks > 0 ? blocks : 1, 256, 0, s>>>(a, g);
    launch_scan_counts(a.countSlot, a.M.ncell, a.scanPartial, a.startB, a.ctl, s);
}

// ---------------------------------------------------------------------------
// rebuild: one warp per cell
// ---------------------------------------------------------------------------
template <typename Real>
__device__ __forceinline__ void copy_particle(const StepArgs<Real>& a, int from, int to)
{
    a.B.x[0][to] = a.A.x[0][from]; a.B.x[1][to] = a.A.x[1][from]; a.B.x[2][to] = a.A.x[2][from];
    a.B.v[0][to] = a.A.v[0][from]; a.B.v[1][to] = a.A.v[1][from]; a.B.v[2][to] = a.A.v[2][from];
    a.B.ir[to] = a.A.ir[from];
}

template <typename Real>
__device__ __forceinline__ void store_position(const StepArgs<Real>& a, int c, int to, const double x[3])
{
    if constexpr (sizeof(Real) == 4) {
        const double* cc = a.M.cellCenter + (size_t)c * 3;
        a.B.x[0][to] = (Real)(x[0] - cc[0]); a.B.x[1][to] = (Real)(x[1] - cc[1]); a.B.x[2][to] = (Real)(x[2] - cc[2]);
    } else {
        a.B.x[0][to] = x[0]; a.B.x[1][to] = x[1]; a.B.x[2][to] = x[2];
    }
}

template <typename Real>
__global__ void __launch_bounds__(256) gsis_rebuild_kernel(StepArgs<Real> a, GsisArgs g)
{
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int c = warp; c < a.M.ncell; c += nwarps) {
        const int sA = a.startA[c], n0 = a.startA[c + 1] - sA;
        const int sB = a.startB[c], n1 = a.startB[c + 1] - sB;
        if (n1 < n0) {
            // deletion (src/ProcessGSIS.cpp:2490-2530): n0 - n1 draws over the
            // shrinking bucket; the last particle moves into the emptied slot.
            // perm[q] is the old index of the particle at bucket position q.
            int* perm = a.idx + sA;
            for (int k = lane; k < n0; k += 32) perm[k] = k;
            __syncwarp();
            if (lane == 0) {
                for (int j = 0; j < n0 - n1; ++j) {
                    const int m = n0 - j;
                    const U4 b = gsis_draw(g, c, j >> 1, 1u, 0u);
                    const int kp = pick_index((j & 1) ? unit64(b.z, b.w) : unit64(b.x, b.y), m);
                    perm[kp] = perm[m - 1];
                }
            }
            __syncwarp();
            for (int q = lane; q < n1; q += 32) copy_particle(a, sA + perm[q], sB + q);
        } else {
            for (int q = lane; q < n0; q += 32) copy_particle(a, sA + q, sB + q);
            const int r = n1 - n0;
            if (r > 0 && n0 == 0) {
                // MaxwellianSample at the NS state (src/ProcessGSIS.cpp:2443-2466)
                const double* ns = g.ns + (size_t)c * 6;
                const double sT = sqrt(ns[4]);
                for (int j = lane; j < r; j += 32) {
                    U4 b[6];
#pragma unroll
                    for (int q = 0; q < 6; ++q) b[q] = gsis_draw(g, c, j, 3u, (uint32_t)q);
                    const int to = sB + j;
#pragma unroll
                    for (int k = 0; k < 3; ++k) {
                        const double rr = unit64(b[k].x, b[k].y);
                        const double th = dm(kTwoPi, unit64(b[k].z, b[k].w));
                        a.B.v[k][to] = (Real)da(dm(dm(sT, sqrt(-log(rr))), sin(th)), ns[1 + k]);
                    }
                    a.B.ir[to] = (Real)dm(dm(-log(unit64(b[3].x, b[3].y)), 0.5), ns[5]);
                    double x[3];
                    place_in_cell(a.M, c, unit64(b[3].z, b[3].w), unit64(b[4].x, b[4].y), unit64(b[4].z, b[4].w),
                                  unit64(b[5].x, b[5].y), unit64(b[5].z, b[5].w), x);
                    store_position(a, c, to, x);
                }
            } else if (r > 0) {
                // replication (src/ProcessGSIS.cpp:2368-2441): copy j picks
                // uniformly among the n0 + j particles of the bucket so far;
                // org[j] is the old particle it copies (copies of copies
                // resolve to the original), then it moves to a random point.
                int* org = a.rank + sB + n0;
                for (int cs = 0; cs < r; cs += 32) {
                    const int j = cs + lane;
                    const bool live = j < r;
                    U4 b0{}, b1{}, b2{};
                    int o = 0, ref = 0;
                    if (live) {
                        b0 = gsis_draw(g, c, j, 2u, 0u);
                        b1 = gsis_draw(g, c, j, 2u, 1u);
                        b2 = gsis_draw(g, c, j, 2u, 2u);
                        const int kp = pick_index(unit64(b0.x, b0.y), n0 + j);
                        if (kp < n0) o = kp;
                        else if (kp - n0 < cs) o = org[kp - n0];
                        else { o = -1; ref = kp - n0 - cs; }   // a lower lane of this round
                    }
                    for (int it = 0; it < 32; ++it) {
                        const int oo = __shfl_sync(kFull, o, ref);
                        if (o < 0) o = oo;
                        if (__all_sync(kFull, o >= 0)) break;
                    }
                    if (live) {
                        org[j] = o;
                        const int from = sA + o, to = sB + n0 + j;
                        a.B.v[0][to] = a.A.v[0][from]; a.B.v[1][to] = a.A.v[1][from]; a.B.v[2][to] = a.A.v[2][from];
                        a.B.ir[to] = a.A.ir[from];
                        double x[3];
                        place_in_cell(a.M, c, unit64(b0.z, b0.w), unit64(b1.x, b1.y), unit64(b1.z, b1.w),
                                      unit64(b2.x, b2.y), unit64(b2.z, b2.w), x);
                        store_position(a, c, to, x);
                    }
                    __syncwarp();
                }
            }
        }
        for (int q = lane; q < n1; q += 32) a.B.cell[sB + q] = c;
        if (g.flag[c] == 0 || n1 == 0) continue;
        __syncwarp();
        // the linear map (src/ProcessGSIS.cpp:2290-2343): sums in bucket order
        double k = 1.0, kr = 1.0, b0 = 0.0, b1 = 0.0, b2 = 0.0;
        if (lane == 0) {
            double n = 0.0, u0 = 0.0, u1 = 0.0, u2 = 0.0, tc = 0.0, trc = 0.0;
            for (int q = sB; q < sB + n1; ++q) {
                const double vx = (double)a.B.v[0][q], vy = (double)a.B.v[1][q], vz = (double)a.B.v[2][q];
                n = da(n, 1.0);
                u0 = da(u0, vx);
                u1 = da(u1, vy);
                u2 = da(u2, vz);
                tc = da(tc, da(da(dm(vx, vx), dm(vy, vy)), dm(vz, vz)));
                trc = da(trc, (double)a.B.ir[q]);
            }
            u0 = __ddiv_rn(u0, n);
            u1 = __ddiv_rn(u1, n);
            u2 = __ddiv_rn(u2, n);
            const double uu = da(da(dm(u0, u0), dm(u1, u1)), dm(u2, u2));
            tc = dm(__ddiv_rn(2.0, dm(3.0, n)), ds(tc, dm(n, uu)));
            trc = dm(__ddiv_rn(__ddiv_rn(4.0, a.C.dr), n), trc);
            const double* ns = g.ns + (size_t)c * 6;
            if (tc > 0.0 && ns[4] > 0.0 && trc > 0.0) {
                k = sqrt(__ddiv_rn(ns[4], tc));
                b0 = ds(ns[1], dm(k, u0));
                b1 = ds(ns[2], dm(k, u1));
                b2 = ds(ns[3], dm(k, u2));
                kr = __ddiv_rn(ns[5], trc);
            }
        }
        k = __shfl_sync(kFull, k, 0);
        kr = __shfl_sync(kFull, kr, 0);
        b0 = __shfl_sync(kFull, b0, 0);
        b1 = __shfl_sync(kFull, b1, 0);
        b2 = __shfl_sync(kFull, b2, 0);
        for (int q = sB + lane; q < sB + n1; q += 32) {
            a.B.v[0][q] = (Real)da(dm(k, (double)a.B.v[0][q]), b0);
            a.B.v[1][q] = (Real)da(dm(k, (double)a.B.v[1][q]), b1);
            a.B.v[2][q] = (Real)da(dm(k, (double)a.B.v[2][q]), b2);
            a.B.ir[q] = (Real)dm(kr, (double)a.B.ir[q]);
        }
        __syncwarp();
    }
}

template <typename Real>
void launch_gsis_rebuild(const StepArgs<Real>& a, const GsisArgs& g, const LaunchShape& L, cudaStream_t s)
{
    gsis_rebuild_kernel<Real><<<L.smCount * 8, 256, 0, s>>>(a, g);
}

template void launch_gsis_count<float>(const StepArgs<float>&, const GsisArgs&, cudaStream_t);
template void launch_gsis_count<double>(const StepArgs<double>&, const GsisArgs&, cudaStream_t);
template void launch_gsis_rebuild<float>(const StepArgs<float>&, const GsisArgs&, const LaunchShape&, cudaStream_t);
template void launch_gsis_rebuild<double>(const StepArgs<double>&, const GsisArgs&, const LaunchShape&, cudaStream_t);

}  // namespace dsmc
