// Device-side building blocks of the DSMC step: case views, Philox streams,
// the exact FP64 ray/triangle test, the guarded FP32 test, and the particle
// tracing loop (ParticleTransportOps::traceParticleDtleft,
// src/ProcessDSMC.cpp:149-221, with CrossboundarySwitch, :1702-1829).
#pragma once

#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

namespace dsmc {

constexpr int kRoleNone = 0;
constexpr int kRoleInterface = 1;
constexpr int kRoleInlet = 2;
constexpr int kRoleOutlet = 3;
constexpr int kRoleWall = 4;
constexpr int kRoleSpecular = 5;

// Trace outcomes (ifout of the reference: 0 stayed, 1 moved, -1 removed).
constexpr int kTraceStay = 0;
constexpr int kTraceMoved = 1;
constexpr int kTraceRemoved = -1;   // left through inlet/outlet
constexpr int kTraceDropped = -2;   // no exit face (reference "Dropped")
constexpr int kTraceLost = -3;      // crossing cap or bad neighbour
constexpr int kNbLost = -100;       // face record: an interface face without a cell on the other side

// Slots of the counting sort (where a particle arrives from, seen from its
// destination cell): 0 itself, 1..6 face neighbour j-1, 7 anything else
// (multi-cell hops and newly injected particles).
constexpr int kFarSlot = 7;
constexpr int kSlots = 8;

// Counter indices (DsmcCounters order, after `steps`).
enum CounterIdx {
    C_INJECTED = 0, C_REMOVED, C_DROPPED, C_LOST, C_WALL_HITS, C_CROSSINGS,
    C_PAIRS, C_COLLISIONS, C_FALLBACKS, C_OVERFLOW, C_BIG_CELLS, C_COUNT
};

// Error bits in the device error word.
constexpr int kErrCapacity = 1;
constexpr int kErrStageCell = 2;   // a cell larger than the stage reached the staged path
constexpr int kErrRejectLoop = 4;
constexpr int kErrSortIndex = 8;
constexpr int kErrGsisCount = 16;  // a GSIS target count outside [0, 2^30)

// Philox RNG stream purposes (third counter word).
constexpr uint32_t kPurposeWall = 1;
constexpr uint32_t kPurposeInject = 2;
constexpr uint32_t kPurposeCollide = 3;
constexpr uint32_t kPurposeFillCount = 4;   // initial fill: per-cell count rounding, counter (cell, 0, 4, 0)
constexpr uint32_t kPurposeFill = 5;        // initial fill: particle k of cell c, counter (c, k, 5, block)
// GSIS particle update: counter (cell, j, 6 | sub << 4 | epoch << 8, block)
// with sub 0 the count rounding, 1 deletion draws, 2 copies, 3 Maxwellian
// samples into empty cells; epoch counts the updates of a case.
constexpr uint32_t kPurposeGsis = 6;

struct DevMesh {
    int ncell, nface, ntri, nwall;
    const int* triOffset;        // [ncell+1]
    const double* triD;          // [ntri*9] A, e1=B-A, e2=C-A (absolute FP64)
    const int2* triFT;           // [ntri] face id, triangle tag
    const unsigned char* faceRole;
    const int2* faceCells;       // [nface] c0, c1 (c1 >= ncell: ghost)
    const int* faceWall;         // [nface] wall slot or -1
    const double* wallRot;       // [nwall*2*9] rotation R(n) for tag 1 (or triangle), tag 2
    const float* wallRotF;       // same, FP32
    const double* cellCenter;    // [ncell*3]
    const double* cellVolume;    // [ncell]
    const int* cell2cell;        // [ncell*6]
    const signed char* revSlot;  // [ncell*6] slot of this cell in neighbour j's list (or -1)
    // face planes (cells with convex[c] != 0): records faceOff[c]..faceOff[c+1]
    const int* faceOff;          // [ncell+1]
    const int4* faceRec;         // face id, index of its first triangle, node count (3/4), and the crossing:
                                 // the cell on the other side (interface), kNbLost, or -(role + 1)
    const float4* planeF;        // outward unit normal, offset relative to the cell centre
    const float4* diagF;         // quads: in-plane normal of the diagonal, offset (relative)
    const double* planeD;        // [nrec*8] n(3), d, m(3), md, absolute
    const unsigned char* convex; // [ncell]
    const float2* recAux;        // [nrec] x: min |e1 x e2| over the record's triangles (0 when one of them is
                                 // ill-conditioned), y: the cell's length scale (sum over axes of the
                                 // largest node offset from the centre)
    int faceStride;              // F when every cell is convex with F records (record k = cell * F + j), else 0
    int allConvex;               // every cell takes the plane path
    // placement tetrahedra of each cell (buildCellInitTets): records
    // placeOff[c]..placeOff[c+1], four vertices each (absolute FP64; the
    // barycentric weights a, b, c, d go to them in this order) and volume
    const int* placeOff;         // [ncell+1]
    const double* placeV;        // [nplace*12]
    const double* placeVol;      // [nplace]
};

struct DevConsts {
    double dtime;
    double twall;        // Twall_ref
    double sqrtTwall;
    double vrms;
    double neff;
    double dtref;
    double omega, eta, alpha, prelax, dr, nref;
    double cdPrefactor;  // collisionDiameterPrefactor, src/ProcessDSMC.cpp:2626-2630
    double expLB;        // 1 / (2.5 - omega): Larsen-Borgnakke energy-fraction exponent
    double invAlpha;     // 1 / alpha: VSS scattering exponent
    float vhsExpF;       // 1 - 2 eta: exponent of the VHS sigma*c ratio (FP32 path)
    float prelaxF;       // P_relax (FP32 path)
    float invPrelaxF;    // 1 / P_relax, 0 when P_relax is 0 (FP32 path)
    uint32_t seedLo, seedHi;
    int maxCross;
    int nss, nscheme, nevery, nrepeat;
    int wallStats;
};

// ---------------------------------------------------------------------------
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
// easy as 1, 2, 3", SC 2011): counter-based, so every draw is a pure
// function of (key, counter) and results do not depend on launch shape.
// ---------------------------------------------------------------------------
struct U4 { uint32_t x, y, z, w; };

__host__ __device__ __forceinline__ uint32_t mulhi32(uint32_t a, uint32_t b)
{
#ifdef __CUDA_ARCH__
    return __umulhi(a, b);
#else
    return (uint32_t)(((uint64_t)a * b) >> 32);
#endif
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0, uint32_t k1)
{
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t lo0 = 0xD2511F53u * c.x;
        const uint32_t hi0 = mulhi32(0xD2511F53u, c.x);
        const uint32_t lo1 = 0xCD9E8D57u * c.z;
        const uint32_t hi1 = mulhi32(0xCD9E8D57u, c.z);
        c = U4{hi1 ^ c.y ^ k0, lo1, hi0 ^ c.w ^ k1, lo0};
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    return c;
}

// Uniform variates from raw Philox words: a double in (0,1) with 53 random
// bits from two words, a float in (0,1) with 24 random bits from one.
__host__ __device__ __forceinline__ double unit64(uint32_t a, uint32_t b)
{
    const uint64_t k = ((uint64_t)a << 21) ^ ((uint64_t)b >> 11);
    return ((double)k + 0.5) * 0x1.0p-53;
}
__device__ __forceinline__ float unit32(uint32_t a) { return ((float)(a >> 8) + 0.5f) * 0x1.0p-24f; }

// A sequential stream over counter (id, step, purpose, n), n = 0, 1, ...
struct Stream {
    uint32_t id, step, purpose, n;
    uint32_t k0, k1;
    U4 buf;
    int avail;

    __device__ __forceinline__ void init(uint32_t id_, uint32_t step_, uint32_t purpose_, uint32_t kLo, uint32_t kHi)
    {
        id = id_; step = step_; purpose = purpose_; n = 0; k0 = kLo; k1 = kHi; avail = 0;
    }
    __device__ __forceinline__ uint32_t next32()
    {
        if (avail == 0) {
            buf = philox4x32_10(U4{id, step, purpose, n}, k0, k1);
            ++n;
            avail = 4;
        }
        const uint32_t r = (avail == 4) ? buf.x : (avail == 3) ? buf.y : (avail == 2) ? buf.z : buf.w;
        --avail;
        return r;
    }
    // uniform double in (0,1) with 53 random bits
    __device__ __forceinline__ double uniform64()
    {
        const uint32_t a = next32();
        const uint32_t b = next32();
        return unit64(a, b);
    }
    // uniform float in (0,1) with 24 random bits
    __device__ __forceinline__ float uniform32() { return unit32(next32()); }
    template <typename Real> __device__ __forceinline__ Real uniform();
};
template <> __device__ __forceinline__ double Stream::uniform<double>() { return uniform64(); }
template <> __device__ __forceinline__ float Stream::uniform<float>() { return uniform32(); }

// The four uniforms of one wall re-emission from a Stream, in order.
template <typename Real>
__device__ __forceinline__ void draw4(Stream& s, const DevConsts&, Real u[4])
{
#pragma unroll
    for (int k = 0; k < 4; ++k) u[k] = s.uniform<Real>();
}

// A stream over counter (id, step, purpose, n) that is only ever drawn a
// whole wall re-emission at a time, starting block-aligned: the same words
// as a Stream drawn the same way (FP32: one block of four words; FP64: two
// blocks, a 53-bit uniform from each pair), kept in one register (n).
struct BlockStream {
    uint32_t id, step, purpose, n;
    __device__ __forceinline__ void init(uint32_t id_, uint32_t step_, uint32_t purpose_)
    {
        id = id_; step = step_; purpose = purpose_; n = 0;
    }
};
template <typename Real>
__device__ __forceinline__ void draw4(BlockStream& s, const DevConsts& C, Real u[4])
{
    if constexpr (sizeof(Real) == 8) {
        const U4 a = philox4x32_10(U4{s.id, s.step, s.purpose, s.n}, C.seedLo, C.seedHi);
        const U4 b = philox4x32_10(U4{s.id, s.step, s.purpose, s.n + 1}, C.seedLo, C.seedHi);
        s.n += 2;
        u[0] = unit64(a.x, a.y); u[1] = unit64(a.z, a.w); u[2] = unit64(b.x, b.y); u[3] = unit64(b.z, b.w);
    } else {
        const U4 a = philox4x32_10(U4{s.id, s.step, s.purpose, s.n}, C.seedLo, C.seedHi);
        s.n += 1;
        u[0] = unit32(a.x); u[1] = unit32(a.y); u[2] = unit32(a.z); u[3] = unit32(a.w);
    }
}

// ---------------------------------------------------------------------------
// Exact FP64 arithmetic helpers: each operation rounded on its own, as the
// reference's x86-64 build evaluates them (no fused multiply-add).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }

// ---------------------------------------------------------------------------
// Placement of new particles (initial fill, GSIS copies and samples)
// ---------------------------------------------------------------------------

// A point of the placement tetrahedron V from four uniforms normalised by
// their sum (randomBarycentric4, src/MeshparticalInitial.cpp:85-106 and
// src/ProcessGSIS.cpp:513-534), out = a V0 + b V1 + c V2 + d V3 evaluated
// left to right (velocityLocationGenerate, src/MeshparticalInitial.cpp:
// 646-721; sampleCellLocation, src/ProcessGSIS.cpp:1000-1028).
__device__ __forceinline__ void place_point(const double* __restrict__ V, double r0, double r1, double r2, double r3,
                                            double out[3])
{
    const double sum = da(da(da(r0, r1), r2), r3);
    double a = 0.25, b = 0.25, c = 0.25, d = 0.25;
    if (sum > 0.0 && isfinite(sum)) {
        a = __ddiv_rn(r0, sum);
        b = __ddiv_rn(r1, sum);
        c = __ddiv_rn(r2, sum);
        d = __ddiv_rn(r3, sum);
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) out[k] = da(da(da(dm(a, V[k]), dm(b, V[3 + k])), dm(c, V[6 + k])), dm(d, V[9 + k]));
}

// sampleCellLocation (src/ProcessGSIS.cpp:977-1029): a placement
// tetrahedron of cell c by volume (the first whose volume is at least the
// remaining pick, subtracting as it goes), then a point in it; the cell
// centre when the cell has no placement tetrahedra (randomlocation's
// fallback, src/ProcessGSIS.cpp:2478-2488).
__device__ __forceinline__ void place_in_cell(const DevMesh& M, int c, double uPick, double r0, double r1, double r2,
                                              double r3, double out[3])
{
    const int t0 = M.placeOff[c], t1 = M.placeOff[c + 1];
    double total = 0.0;
    for (int t = t0; t < t1; ++t) total = da(total, M.placeVol[t]);
    if (t1 <= t0 || !(total > 0.0) || !isfinite(total)) {
        out[0] = M.cellCenter[(size_t)c * 3 + 0];
        out[1] = M.cellCenter[(size_t)c * 3 + 1];
        out[2] = M.cellCenter[(size_t)c * 3 + 2];
        return;
    }
    double pick = dm(uPick, total);
    int ch = t1 - 1;
    for (int t = t0; t < t1; ++t) {
        const double v = M.placeVol[t];
        if (pick <= v) { ch = t; break; }
        pick = ds(pick, v);
    }
    place_point(M.placeV + (size_t)ch * 12, r0, r1, r2, r3, out);
}

// intersectCachedTri, src/ProcessDSMC.cpp:1174-1197, operation for operation.
__device__ __forceinline__ bool isect_exact(const double* __restrict__ T, const double x[3], const double v[3], double& t)
{
    const double ax = T[0], ay = T[1], az = T[2];
    const double e1x = T[3], e1y = T[4], e1z = T[5];
    const double e2x = T[6], e2y = T[7], e2z = T[8];
    const double p0 = ds(dm(v[1], e2z), dm(v[2], e2y));
    const double p1 = ds(dm(v[2], e2x), dm(v[0], e2z));
    const double p2 = ds(dm(v[0], e2y), dm(v[1], e2x));
    const double det = da(da(dm(e1x, p0), dm(e1y, p1)), dm(e1z, p2));
    if (fabs(det) < 1e-14) return false;
    const double inv = __ddiv_rn(1.0, det);
    const double t0 = ds(x[0], ax), t1 = ds(x[1], ay), t2 = ds(x[2], az);
    const double u = dm(da(da(dm(t0, p0), dm(t1, p1)), dm(t2, p2)), inv);
    if (u < 0.0 || u > 1.0) return false;
    const double q0 = ds(dm(t1, e1z), dm(t2, e1y));
    const double q1 = ds(dm(t2, e1x), dm(t0, e1z));
    const double q2 = ds(dm(t0, e1y), dm(t1, e1x));
    const double vv = dm(da(da(dm(v[0], q0), dm(v[1], q1)), dm(v[2], q2)), inv);
    if (vv < 0.0 || da(u, vv) > 1.0) return false;
    t = dm(da(da(dm(e2x, q0), dm(e2y, q1)), dm(e2z, q2)), inv);
    return t > 1e-14;
}

struct ExitHit {
    int face;   // -2: none
    int tri;
    double t;
};

// tryCachedCellIntersection, src/ProcessDSMC.cpp:1210-1251. The reference's
// uncached fallback (intersectFallbackCell, :1484-1524) repeats the same
// products and sums on the same node coordinates, so it cannot find a hit the
// cached test missed; a miss here is a miss there. Triangles of the entry face
// are skipped by the reference's rule (:1229-1233): all of a triangular face,
// only the same half of a quad.
__device__ __forceinline__ ExitHit find_exit_exact(const DevMesh& M, int cell, int crossf, int prevTri,
                                                   const double x[3], const double v[3])
{
    ExitHit h{-2, -1, DBL_MAX};
    const int b = M.triOffset[cell];
    const int e = M.triOffset[cell + 1];
    for (int k = b; k < e; ++k) {
        const int2 ft = M.triFT[k];
        if (ft.x == crossf) {
            if (ft.y <= 0 || (prevTri != 1 && prevTri != 2) || ft.y == prevTri) continue;
        }
        double t = DBL_MAX;
        if (isect_exact(M.triD + (size_t)k * 9, x, v, t) && t < h.t) {
            h.t = t;
            h.face = ft.x;
            h.tri = ft.y;
        }
    }
    if (h.face == -2) h.t = DBL_MAX;
    return h;
}

// ---------------------------------------------------------------------------
// Plane-based exit search of the FP64 path, for cells that are convex with
// planar faces.
//
// The exit of a ray from inside a convex cell is the face plane it reaches
// first among those it moves towards: t_f = (d_f - n_f.x) / (v.n_f) for
// v.n_f > 0. That takes one dot-product pair per face instead of a full
// triangle test per triangle. The result is only trusted when it is clear of
// every tie the triangle tests could resolve differently: a second plane
// reached within the error bound (edge or vertex), a tiny or negative t, a
// position on, outside or within twice the error bound of any face plane
// other than the entry face's, and for quads a hit point within the bound of
// the split diagonal
// (which sub-triangle). Otherwise `ambiguous` is set and the caller runs the
// triangle search. The entry face (crossf) is never the exit: the particle
// sits on it and moves away from it.
// ---------------------------------------------------------------------------
struct PlaneHit {
    int face;
    int tri;       // -1 triangle face, 1/2 quad half
    int triIdx;    // index of that triangle in the cell's triangle list
    double t;
    bool ambiguous;
    int nb;        // the record's crossing: the cell on the other side, kNbLost or -(role + 1)
};

__device__ __forceinline__ PlaneHit find_exit_planes(const DevMesh& M, int cell, int crossf, const double x[3],
                                                     const double v[3])
{
    constexpr double eps = 1.1102230246251565e-16;
    constexpr double K = 64;
    PlaneHit h{-2, -1, -1, 0.0, false, 0};
    const double vnorm = fabs(v[0]) + fabs(v[1]) + fabs(v[2]);
    const double xnorm = fabs(x[0]) + fabs(x[1]) + fabs(x[2]);
    double best = DBL_MAX, second = DBL_MAX, bestErr = 0, secondErr = 0;
    int bi = -1;
    bool amb = false;
    const int b = M.faceStride ? cell * M.faceStride : M.faceOff[cell];
    const int e = M.faceStride ? b + M.faceStride : M.faceOff[cell + 1];
    for (int k = b; k < e; ++k) {
        const int4 rec = M.faceRec[k];
        if (rec.x == crossf) continue;
        const double* pd = M.planeD + (size_t)k * 8;
        const double nx = pd[0], ny = pd[1], nz = pd[2], d = pd[3];
        const double vn = v[0] * nx + v[1] * ny + v[2] * nz;
        const double num = d - (x[0] * nx + x[1] * ny + x[2] * nz);
        const double dErr = K * eps * (fabs(d) + xnorm);
        const double vErr = K * eps * vnorm;
        // on, outside or within the error bound of a face it did not enter
        // through: the reference's test of that face's triangles can see a
        // hit at t ~ 0 (a start on a vertex, an edge or a face)
        if (num <= 2.0 * dErr) amb = true;
        if (vn <= vErr) continue;
        const double t = num / vn;
        const double tErr = (dErr + fabs(t) * vErr) / vn;
        if (t < best) {
            second = best; secondErr = bestErr;
            best = t; bestErr = tErr; bi = k;
        } else if (t < second) {
            second = t; secondErr = tErr;
        }
    }
    if (bi < 0) { h.ambiguous = true; return h; }
    if (best <= bestErr) amb = true;
    if (second - best <= bestErr + secondErr) amb = true;
    const int4 rec = M.faceRec[bi];
    h.face = rec.x;
    h.t = best;
    h.tri = -1;
    h.triIdx = rec.y;
    h.nb = rec.w;
    if (rec.z == 4) {
        const double* pd = M.planeD + (size_t)bi * 8;
        const double mx = pd[4], my = pd[5], mz = pd[6], md = pd[7];
        const double px = x[0] + v[0] * best, py = x[1] + v[1] * best, pz = x[2] + v[2] * best;
        const double side = mx * px + my * py + mz * pz - md;
        const double sErr = K * eps * (fabs(md) + fabs(px) + fabs(py) + fabs(pz)) + vnorm * bestErr;
        if (fabs(side) <= sErr) amb = true;
        h.tri = side > 0.0 ? 1 : 2;
        h.triIdx = rec.y + (h.tri == 2 ? 1 : 0);
    }
    h.ambiguous = amb;
    return h;
}

// ---------------------------------------------------------------------------
// The mixed path's exit test: FP32 arithmetic that settles, where it can, what
// the reference's FP64 triangle scan (find_exit_exact) returns, so that the
// mixed trace takes the same decisions as the FP64 trace.
//
// Inputs: the position relative to the cell centre rounded to FP32 from the
// trace's FP64 position, the FP32 velocity, and the cell's FP32 face planes.
// Every quantity carries a bound on its error: dErr on a plane distance
// (32 ulp of the operands' size plus the cell's length scale, five times the
// worst case of the roundings in x, n, d and the dot product, and far above
// the reference's own FP64 rounding in absolute coordinates), vErr on v.n.
// The result is `certain` when:
//   - every face other than the entry face is either approached (v.n > vErr)
//     or left behind (v.n < -vErr), with the particle inside its plane by
//     more than twice its dErr (so no face test can see a hit behind the
//     particle or at t ~ 0);
//   - the approached face f reached first is reached, within its interval
//     [tLo, tHi], before any other approached face could be, with a margin
//     of one dErr at the hit point on every other face's plane, the entry
//     face's included: the hit point lies inside f's triangle by more than
//     the FP64 test's rounding, and no other triangle's hit can come first;
//   - f is neither grazed (v.n_f below 2^-10 |v|) nor ill-conditioned, and
//     its triangles' determinants stay above the reference's 1e-14 cut;
//   - for a quad f, the hit point is clear of the split diagonal (which half),
//     and after entering through half `tag` of a quad, the position is clear
//     of that face's diagonal on the side of `tag` (the reference still tests
//     the other half, :1229-1233; it cannot hit from there).
// Then the reference's scan returns f (with the half `tri`) at a t inside
// [tLo, tHi]. Anything else is not certain and the caller runs that scan.
// ---------------------------------------------------------------------------
struct CertainExit {
    bool certain;
    int face, tri, triIdx;
    int nb;        // the record's crossing (as PlaneHit::nb)
    float tLo, tHi;
};

constexpr float kEps32 = 5.9604645e-8f;   // 2^-24

// kAtRest: the search of a particle at rest in its cell (crossf -1, as in
// the stay pass), which has no entry face and reads no face records in its
// loop; the same result as the general form with crossf -1.
// kFaces > 0: the mesh's face records sit at cell * kFaces (faceStride ==
// kFaces, checked by the caller), and the face loop is unrolled with its
// loads issued together.
template <bool kAtRest = false, int kFaces = 0>
__device__ __forceinline__ CertainExit certain_exit_f32(const DevMesh& M, int cell, int crossf, int tag,
                                                        const float x[3], const float v[3], float absScale)
{
    CertainExit r{false, -2, -1, -1, 0, 0.0f, 0.0f};
    const float vnorm = fabsf(v[0]) + fabsf(v[1]) + fabsf(v[2]);
    const float xnorm = fabsf(x[0]) + fabsf(x[1]) + fabsf(x[2]);
    const float vErr = 32.0f * kEps32 * vnorm;
    const float absErr = 0x1p-30f * absScale;
    const int b = kFaces ? cell * kFaces : (M.faceStride ? cell * M.faceStride : M.faceOff[cell]);
    const int e = kFaces ? b + kFaces : (M.faceStride ? b + M.faceStride : M.faceOff[cell + 1]);
    int bi = -1;
    float best = FLT_MAX, bestLo = 0.0f, bestHi = 0.0f, bestTau = 0.0f, bestVn = 0.0f;
    float tauMin = FLT_MAX;   // latest t_f every other approached face allows
    float entA = 0.0f, entB = 0.0f;
    bool ok = true;
    // the length scale is the cell's (the same in each of its records)
    const float lc = b < e ? M.recAux[b].y : 0.0f;
    const float dErr0 = 32.0f * kEps32 * (xnorm + lc) + absErr;
#pragma unroll(kFaces > 0 ? kFaces : 1)
    for (int k = b; k < e; ++k) {
        int4 rec = make_int4(-1, 0, 0, 0);
        if constexpr (!kAtRest) rec = M.faceRec[k];
        const float4 pl = M.planeF[k];
        const float vn = v[0] * pl.x + v[1] * pl.y + v[2] * pl.z;
        const float num = pl.w - (x[0] * pl.x + x[1] * pl.y + x[2] * pl.z);
        const float dErr = 32.0f * kEps32 * fabsf(pl.w) + dErr0;
        if (!kAtRest && rec.x == crossf) {
            // entry face: moving away from it; its edge with the exit face is
            // checked below (slack entA + t_f * entB)
            if (!(vn < -vErr)) ok = false;
            entA = num - 2.0f * dErr;
            entB = -vn - vErr;
            if (rec.z == 4 && (tag == 1 || tag == 2)) {
                const float4 dg = M.diagF[k];
                const float side = dg.x * x[0] + dg.y * x[1] + dg.z * x[2] - dg.w;
                const float sErr = 2.0f * (32.0f * kEps32 * (fabsf(dg.w) + xnorm + lc) + absErr);
                if (!(tag == 1 ? side > sErr : side < -sErr)) ok = false;
            }
            continue;
        }
        if (!(num > 2.0f * dErr) || !(fabsf(vn) > vErr)) { ok = false; continue; }
        if (vn < 0.0f) continue;   // left behind: never reached
        // fast divisions (a few ulp, well inside dErr's margin), each bound
        // then moved outwards by 2^-21 of itself
        const float t = __fdividef(num, vn);
        const float tLo = __fdividef(num - dErr, vn + vErr) * (1.0f - 0x1p-21f);
        const float tHi = __fdividef(num + dErr, vn - vErr) * (1.0f + 0x1p-21f);
        const float tau = __fdividef(num - 2.0f * dErr, vn + vErr) * (1.0f - 0x1p-21f);
        if (t < best) {
            if (bi >= 0) tauMin = fminf(tauMin, bestTau);
            best = t; bestLo = tLo; bestHi = tHi; bestTau = tau; bestVn = vn; bi = k;
        } else {
            tauMin = fminf(tauMin, tau);
        }
    }
    if (!ok || bi < 0) return r;
    if (!(bestHi < tauMin)) return r;
    if (crossf >= 0 && !(entA + bestLo * entB > 0.0f)) return r;
    const float2 aux = M.recAux[bi];
    if (!(bestVn >= 0x1p-10f * vnorm)) return r;            // grazing exit
    if (!((bestVn - vErr) * aux.x > 2e-14f)) return r;       // |det| near the 1e-14 cut, or ill-conditioned
    if (!(bestLo > 2e-14f)) return r;                        // the reference's t > 1e-14
    const int4 rec = M.faceRec[bi];
    int tri = -1, triIdx = rec.y;
    if (rec.z == 4) {
        const float4 dg = M.diagF[bi];
        const float px = x[0] + v[0] * best, py = x[1] + v[1] * best, pz = x[2] + v[2] * best;
        const float side = dg.x * px + dg.y * py + dg.z * pz - dg.w;
        const float sErr = 32.0f * kEps32 * (fabsf(dg.w) + fabsf(px) + fabsf(py) + fabsf(pz) + aux.y) + absErr +
                           vnorm * (bestHi - bestLo);
        if (!(fabsf(side) > 2.0f * sErr)) return r;
        tri = side > 0.0f ? 1 : 2;
        triIdx = rec.y + (tri == 2 ? 1 : 0);
    }
    r.certain = true;
    r.face = rec.x;
    r.tri = tri;
    r.triIdx = triIdx;
    r.nb = rec.w;
    r.tLo = bestLo;
    r.tHi = bestHi;
    return r;
}

// ---------------------------------------------------------------------------
// Particle state in registers and the tracing loop.
// ---------------------------------------------------------------------------
// Positions are absolute FP64 while a particle is traced, in both paths: the
// mixed path stores them in HBM as FP32 offsets from the cell centre and
// widens them on load (centre + offset, one rounding), so its trace advances
// exactly the positions the FP64 trace would from the same stored state.
template <typename Real>
struct PRegs {
    double x[3];
    Real v[3];
    Real ir;
};

struct TraceLog {        // optional per-particle record for the tracing check
    int hitFace;
    int hitTri;
    int ncross;
};

struct WallTally {
    double* tally;       // [nwall*6] or nullptr
};

// Diffuse re-emission at a wall (CrossboundarySwitch Wall case,
// src/ProcessDSMC.cpp:1793-1825): Maxwellian at Twall_ref in the local frame
// of the wall normal, rotational energy -ln(r) Tw / 2.
template <typename Real, typename Rng>
__device__ __forceinline__ void diffuse_reflect(const DevMesh& M, const DevConsts& C, int wslot, int tag,
                                                PRegs<Real>& p, Rng& rng)
{
    const int which = (tag == 2) ? 1 : 0;
    Real u[4];
    draw4<Real>(rng, C, u);
    const Real r1 = u[0], r2 = u[1], al = u[2], r3 = u[3];
    Real s, c;
    if constexpr (sizeof(Real) == 8) {
        sincospi(2.0 * al, &s, &c);
        const double* R = M.wallRot + ((size_t)wslot * 2 + which) * 9;
        const double st = C.sqrtTwall;
        const double a = sqrt(-log(r2));
        const double vxp = a * s * st;
        const double vyp = a * c * st;
        const double vzp = -sqrt(-log(r1)) * st;
        p.v[0] = R[0] * vxp + R[1] * vyp + R[2] * vzp;
        p.v[1] = R[3] * vxp + R[4] * vyp + R[5] * vzp;
        p.v[2] = R[6] * vxp + R[7] * vyp + R[8] * vzp;
        p.ir = -log(r3) * C.twall * 0.5;
    } else {
        sincospif(2.0f * al, &s, &c);
        const float* R = M.wallRotF + ((size_t)wslot * 2 + which) * 9;
        const float st = (float)C.sqrtTwall;
        const float a = sqrtf(-__logf(r2));
        const float vxp = a * s * st;
        const float vyp = a * c * st;
        const float vzp = -sqrtf(-__logf(r1)) * st;
        p.v[0] = R[0] * vxp + R[1] * vyp + R[2] * vzp;
        p.v[1] = R[3] * vxp + R[4] * vyp + R[5] * vzp;
        p.v[2] = R[6] * vxp + R[7] * vyp + R[8] * vzp;
        p.ir = -__logf(r3) * (float)C.twall * 0.5f;
    }
}

// Mirror reflection about the wall normal (third column of R); no reference
// counterpart (the reference leaves such tags unmapped).
template <typename Real>
__device__ __forceinline__ void specular_reflect(const DevMesh& M, int wslot, int tag, PRegs<Real>& p)
{
    const int which = (tag == 2) ? 1 : 0;
    Real n0, n1, n2;
    if constexpr (sizeof(Real) == 8) {
        const double* R = M.wallRot + ((size_t)wslot * 2 + which) * 9;
        n0 = R[2]; n1 = R[5]; n2 = R[8];
    } else {
        const float* R = M.wallRotF + ((size_t)wslot * 2 + which) * 9;
        n0 = R[2]; n1 = R[5]; n2 = R[8];
    }
    const Real vn = p.v[0] * n0 + p.v[1] * n1 + p.v[2] * n2;
    p.v[0] -= 2 * vn * n0;
    p.v[1] -= 2 * vn * n1;
    p.v[2] -= 2 * vn * n2;
}

// Counters accumulated per thread and flushed once per warp.
struct TraceCounts {
    uint32_t removed, dropped, lost, wall, cross, fallback;
};

// x += v t (scalar_product, src/ProcessDSMC.cpp:1611-1617), in FP64 with
// each operation rounded on its own (an FP32 velocity widens exactly)
template <typename Real>
__device__ __forceinline__ void advance(PRegs<Real>& p, double t)
{
#pragma unroll
    for (int d = 0; d < 3; ++d) p.x[d] = da(p.x[d], dm((double)p.v[d], t));
}

// The tracing loop's state between two exit searches.
struct TraceState {
    int ifout;        // outcome so far
    int iter;         // exit searches made
    int crossf, tag;  // the face / triangle the particle entered through
    bool afterNone;   // the last hit had no handler: use the triangle search
    __device__ __forceinline__ void begin(int crossf0, int tag0)
    {
        ifout = kTraceStay;
        iter = 0;
        crossf = crossf0;
        tag = tag0;
        afterNone = false;
    }
};

// One pass of the tracing loop (traceParticleDtleft, src/ProcessDSMC.cpp:
// 149-221): an exit search from `cell` and either the advance to the end of
// the step or the crossing with its boundary handling. Returns true when the
// trace is over, with the outcome in st.ifout.
//
// Exit search. FP64 path: the FP64 plane decision confirmed by the
// reference's test on the chosen triangle, else the reference's triangle
// scan. Mixed path: certain_exit_f32 on the FP32 offsets; a certain exit
// beyond the rest of the step needs no FP64 test at all (the particle stays),
// a certain crossing takes its t from the reference's FP64 test on the one
// triangle it names, and everything else runs the reference's FP64 triangle
// scan (counter `fp64_fallbacks`). Positions, dtleft and every decision are
// then those of the FP64 trace from the same stored state; only wall
// re-emission draws FP32 velocities.
template <typename Real, typename Rng>
__device__ __forceinline__ bool trace_step(const DevMesh& M, const DevConsts& C, PRegs<Real>& p, int& cell,
                                           double& dtleft, TraceState& st, Rng& rng, int istep,
                                           double* wallTally, TraceCounts& cnt, bool stopAtWall, TraceLog* log)
{
    int& ifout = st.ifout;
    int& crossf = st.crossf;
    int& tag = st.tag;
    bool& afterNone = st.afterNone;
    if (!(dtleft > 0.0)) return true;
    if (st.iter++ >= C.maxCross) { cnt.lost++; dtleft = 0; ifout = kTraceLost; return true; }
    int face = -2, tri = -1;
    double t = 0.0;
    bool decided = false;
    int hintNb = 0;   // a face chosen from a face record comes with the record's crossing
    if ((M.allConvex || M.convex[cell]) && !afterNone) {
        if constexpr (sizeof(Real) == 8) {
            // plane decision, then the reference's exact test on that one
            // triangle for the bit-exact t; any doubt runs the full search
            const PlaneHit ph = find_exit_planes(M, cell, crossf, p.x, p.v);
            double te = DBL_MAX;
            if (!ph.ambiguous && isect_exact(M.triD + (size_t)ph.triIdx * 9, p.x, p.v, te)) {
                face = ph.face; tri = ph.tri; t = te;
                decided = true;
                hintNb = ph.nb;
                // the other half of a quad entry face stays eligible in
                // the reference's skip rule (src/ProcessDSMC.cpp:1229-1233)
                if (crossf >= 0 && (tag == 1 || tag == 2)) {
                    const int b0 = M.triOffset[cell], e0 = M.triOffset[cell + 1];
                    for (int k = b0; k < e0; ++k) {
                        const int2 ft = M.triFT[k];
                        if (ft.x != crossf || ft.y == tag || ft.y <= 0) continue;
                        double t2 = DBL_MAX;
                        if (isect_exact(M.triD + (size_t)k * 9, p.x, p.v, t2) && t2 < t) decided = false;
                    }
                }
            }
        } else {
            const double* cc = M.cellCenter + (size_t)cell * 3;
            const double c0 = cc[0], c1 = cc[1], c2 = cc[2];
            const float xr[3] = {(float)ds(p.x[0], c0), (float)ds(p.x[1], c1), (float)ds(p.x[2], c2)};
            const float absScale = (float)(fabs(c0) + fabs(c1) + fabs(c2));
            const CertainExit ce = M.faceStride == 4
                                       ? certain_exit_f32<false, 4>(M, cell, crossf, tag, xr, p.v, absScale)
                                       : certain_exit_f32<false, 0>(M, cell, crossf, tag, xr, p.v, absScale);
            if (ce.certain) {
                if (ce.tLo > (float)dtleft * (1.0f + 0x1p-16f)) {
                    // the reference's scan would return this face at t >= dtleft
                    advance(p, dtleft);
                    dtleft = 0;
                    return true;
                }
                const double v64[3] = {(double)p.v[0], (double)p.v[1], (double)p.v[2]};
                double te = DBL_MAX;
                if (isect_exact(M.triD + (size_t)ce.triIdx * 9, p.x, v64, te)) {
                    face = ce.face; tri = ce.tri; t = te;
                    decided = true;
                    hintNb = ce.nb;
                }
            }
        }
    }
    if constexpr (sizeof(Real) == 4) {
        if (!decided) cnt.fallback++;
    }
    if (!decided) {
        const double v64[3] = {(double)p.v[0], (double)p.v[1], (double)p.v[2]};
        const ExitHit h = find_exit_exact(M, cell, crossf, tag, p.x, v64);
        if (h.face == -2 || !isfinite(h.t) || h.t <= 0.0) { cnt.dropped++; dtleft = 0; ifout = kTraceDropped; return true; }
        face = h.face; tri = h.tri; t = h.t;
    }
    if (t >= dtleft) {
        advance(p, dtleft);
        dtleft = 0;
        return true;
    }
    crossf = face;
    tag = tri;
    const int role = !decided ? (int)M.faceRole[face] : (hintNb >= 0 || hintNb == kNbLost) ? kRoleInterface : -(hintNb + 1);
    if (log && role != kRoleInterface && log->hitFace < 0) {
        log->hitFace = face;
        log->hitTri = tri;
        if (stopAtWall && role == kRoleWall) {
            advance(p, t);
            dtleft = ds(dtleft, t);
            return true;
        }
    }
    cnt.cross++;
    if (log) log->ncross++;
    // x += v t (scalar_product, src/ProcessDSMC.cpp:1611-1617) for every
    // role that has a handler
    if (role != kRoleNone) advance(p, t);
    if (role == kRoleInterface) {
        ifout = kTraceMoved;
        dtleft = ds(dtleft, t);
        int next;
        if (decided) {
            next = hintNb;
        } else {
            const int2 cc = M.faceCells[face];
            if (cell == cc.x) next = cc.y;
            else if (cell == cc.y) next = cc.x;
            else next = cc.x;
        }
        if (next < 0 || next >= M.ncell) { cnt.lost++; dtleft = 0; ifout = kTraceLost; return true; }
        cell = next;
    } else if (role == kRoleInlet || role == kRoleOutlet) {
        cnt.removed++;
        dtleft = 0;
        ifout = kTraceRemoved; return true;
    } else if (role == kRoleWall) {
        dtleft = ds(dtleft, t);
        const int ws = M.faceWall[face];
        const Real v0 = p.v[0], v1 = p.v[1], v2 = p.v[2], ir0 = p.ir;
        diffuse_reflect<Real, Rng>(M, C, ws, tri, p, rng);
        cnt.wall++;
        if (wallTally && C.wallStats && istep > C.nss) {
            double* T = wallTally + (size_t)ws * 6;
            const double a0 = (double)p.v[0], a1 = (double)p.v[1], a2 = (double)p.v[2];
            const double b0 = (double)v0, b1 = (double)v1, b2 = (double)v2;
            atomicAdd(T + 0, 1.0);
            atomicAdd(T + 1, a0 - b0);
            atomicAdd(T + 2, a1 - b1);
            atomicAdd(T + 3, a2 - b2);
            atomicAdd(T + 4, 0.5 * ((a0 * a0 + a1 * a1 + a2 * a2) - (b0 * b0 + b1 * b1 + b2 * b2)));
            atomicAdd(T + 5, (double)p.ir - (double)ir0);
        }
    } else if (role == kRoleSpecular) {
        dtleft = ds(dtleft, t);
        specular_reflect<Real>(M, M.faceWall[face], tri, p);
        cnt.wall++;
    }
    // kRoleNone: no handler (src/ProcessDSMC.cpp:1826-1827); the next
    // search excludes this face and the particle is dropped.
    afterNone = (role == kRoleNone);
    return false;
}

// The first exit search of a particle at rest in `cell` at the start of the
// step (no entry face), taken only when it settles that the particle stays
// in its cell for the whole of dtleft: the decision trace_step takes on that
// search, without the triangle scan. The caller then advances it by dtleft.
// FP64 path: the plane decision and the reference's test on the chosen
// triangle; mixed path: certain_exit_f32.
template <typename Real>
__device__ __forceinline__ bool stays_for_the_step(const DevMesh& M, int cell, const PRegs<Real>& p, double dtleft)
{
    if (!(M.allConvex || M.convex[cell])) return false;
    if constexpr (sizeof(Real) == 8) {
        const PlaneHit ph = find_exit_planes(M, cell, -1, p.x, p.v);
        double te = DBL_MAX;
        return !ph.ambiguous && isect_exact(M.triD + (size_t)ph.triIdx * 9, p.x, p.v, te) && te >= dtleft;
    } else {
        const double* cc = M.cellCenter + (size_t)cell * 3;
        const double c0 = cc[0], c1 = cc[1], c2 = cc[2];
        const float xr[3] = {(float)ds(p.x[0], c0), (float)ds(p.x[1], c1), (float)ds(p.x[2], c2)};
        const float absScale = (float)(fabs(c0) + fabs(c1) + fabs(c2));
        const CertainExit ce = M.faceStride == 4 ? certain_exit_f32<true, 4>(M, cell, -1, -1, xr, p.v, absScale)
                                                 : certain_exit_f32<true, 0>(M, cell, -1, -1, xr, p.v, absScale);
        return ce.certain && ce.tLo > (float)dtleft * (1.0f + 0x1p-16f);
    }
}

// Trace one particle, starting in `cell` having entered through face
// `crossf` / triangle `tag` (-1/-1 for a particle at rest in its cell), for
// `dtleft` (updated: the time not flown when the trace stops). Returns the
// reference's outcome and leaves the final cell in `cell`.
template <typename Real>
__device__ int trace_particle(const DevMesh& M, const DevConsts& C, PRegs<Real>& p, int& cell,
                             int crossf, int tag, double& dtleft, Stream& rng, int istep,
                             double* wallTally, TraceCounts& cnt, bool stopAtWall, TraceLog* log)
{
    TraceState st;
    st.begin(crossf, tag);
    while (!trace_step<Real, Stream>(M, C, p, cell, dtleft, st, rng, istep, wallTally, cnt, stopAtWall, log)) {
    }
    return st.ifout;
}

// Warp-aggregated atomic claim of `n` consecutive slots in counter[key];
// returns this lane's slot. Lanes with key < 0 take no slot. The whole warp
// must call it together (full mask).
__device__ __forceinline__ int warp_claim(int* counter, int key)
{
    const unsigned peers = __match_any_sync(0xffffffffu, key);
    const int lane = threadIdx.x & 31;
    const int leader = __ffs(peers) - 1;
    int base = 0;
    if (key >= 0 && lane == leader) base = atomicAdd(counter + key, __popc(peers));
    base = __shfl_sync(0xffffffffu, base, leader);
    return base + __popc(peers & ((1u << lane) - 1u));
}

__device__ __forceinline__ void flush_counts(unsigned long long* ctr, const TraceCounts& c)
{
    uint32_t v[6] = {c.removed, c.dropped, c.lost, c.wall, c.cross, c.fallback};
    const int idx[6] = {C_REMOVED, C_DROPPED, C_LOST, C_WALL_HITS, C_CROSSINGS, C_FALLBACKS};
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        uint32_t s = v[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if ((threadIdx.x & 31) == 0 && s) atomicAdd(ctr + idx[k], (unsigned long long)s);
    }
}

}  // namespace dsmc
