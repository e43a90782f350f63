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
    const float4* triF;          // [ntri*3] A-centre(3) e1(3) e2(3) |e1||e2| face tag (FP32)
    const unsigned char* faceRole;
    const int2* faceCells;       // [nface] c0, c1 (c1 >= ncell: ghost)
    const float4* faceDelta;     // [nface] centre(c0) - centre(c1) as FP32
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
    const float4* nbDeltaF;      // [nrec] FP32 centre shift of a crossing through the record (this - other)
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
// cached test missed; a miss here is a miss there.
//
// entryFace / posTol serve the mixed path only: its positions carry FP32
// rounding, so a particle sitting on the face it entered through can see
// that face again at a tiny positive t that the reference, with exact
// positions, rejects through its 1e-14 cut. Hits on entryFace closer than
// posTol / |v.n| are therefore treated as on the face (no hit).
__device__ __forceinline__ ExitHit find_exit_exact(const DevMesh& M, int cell, int crossf, int prevTri,
                                                   const double x[3], const double v[3],
                                                   int entryFace = -1, double posTol = 0.0)
{
    ExitHit h{-2, -1, DBL_MAX};
    const int b = M.triOffset[cell];
    const int e = M.triOffset[cell + 1];
    for (int k = b; k < e; ++k) {
        const int2 ft = M.triFT[k];
        if (ft.x == crossf) {
            if (ft.y <= 0 || (prevTri != 1 && prevTri != 2) || ft.y == prevTri) continue;
        }
        const double* T = M.triD + (size_t)k * 9;
        double t = DBL_MAX;
        if (isect_exact(T, x, v, t) && t < h.t) {
            if (ft.x == entryFace) {
                const double nx = T[4] * T[8] - T[5] * T[7];
                const double ny = T[5] * T[6] - T[3] * T[8];
                const double nz = T[3] * T[7] - T[4] * T[6];
                const double vn = fabs(v[0] * nx + v[1] * ny + v[2] * nz) / sqrt(nx * nx + ny * ny + nz * nz);
                if (t * vn <= posTol) continue;
            }
            h.t = t;
            h.face = ft.x;
            h.tri = ft.y;
        }
    }
    if (h.face == -2) h.t = DBL_MAX;
    return h;
}

// Guarded FP32 exit search. Positions are relative to the cell centre, so
// x - A carries no cancellation from the domain's absolute coordinates.
// Every decision the reference takes (|det| against 1e-14, u/v/u+v against
// [0,1], t against 1e-14, the smallest t, t against dtleft) is taken in FP32
// only when the FP32 value is farther from the threshold than an error bound
// K*eps32/rel_det (rel_det = |det| / (|e1||e2||v|)); otherwise `ambiguous` is
// set and the caller repeats the step in exact FP64.
struct ExitHitF {
    int face;
    int tri;
    float t;
    float terr;
    bool ambiguous;
};

constexpr float kGuardK = 256.0f * 5.9604645e-8f;   // 256 ulp(1) of FP32

__device__ __forceinline__ ExitHitF find_exit_f32(const DevMesh& M, int cell, int crossf, int prevTri,
                                                   const float x[3], const float v[3], float vnorm,
                                                   int entryFace, float posTol)
{
    ExitHitF h{-2, -1, FLT_MAX, 0.0f, false};
    float second = FLT_MAX, secondErr = 0.0f;
    const int b = M.triOffset[cell];
    const int e = M.triOffset[cell + 1];
    for (int k = b; k < e; ++k) {
        const float4 r0 = M.triF[(size_t)k * 3 + 0];
        const float4 r1 = M.triF[(size_t)k * 3 + 1];
        const float4 r2 = M.triF[(size_t)k * 3 + 2];
        const int face = __float_as_int(r2.z);
        const int tag = __float_as_int(r2.w);
        if (face == crossf) {
            if (tag <= 0 || (prevTri != 1 && prevTri != 2) || tag == prevTri) continue;
        }
        const float ax = r0.x, ay = r0.y, az = r0.z;
        const float e1x = r0.w, e1y = r1.x, e1z = r1.y;
        const float e2x = r1.z, e2y = r1.w, e2z = r2.x;
        const float e12 = r2.y;
        const float p0 = v[1] * e2z - v[2] * e2y;
        const float p1 = v[2] * e2x - v[0] * e2z;
        const float p2 = v[0] * e2y - v[1] * e2x;
        const float det = e1x * p0 + e1y * p1 + e1z * p2;
        const float scale = e12 * vnorm;               // |e1||e2||v|
        const float adet = fabsf(det);
        if (!(adet > 1e-6f * scale) || adet < 1e-13f) {
            // near-parallel ray, degenerate triangle or |det| near the
            // reference's absolute 1e-14 cut: FP32 cannot decide
            if (scale > 0.0f) h.ambiguous = true;
            continue;
        }
        const float inv = 1.0f / det;
        const float err = kGuardK * scale * fabsf(inv);  // bound on |u|,|v| errors
        const float t0 = x[0] - ax, t1 = x[1] - ay, t2 = x[2] - az;
        const float u = (t0 * p0 + t1 * p1 + t2 * p2) * inv;
        if (u < -err || u > 1.0f + err) continue;      // certain miss
        const float q0 = t1 * e1z - t2 * e1y;
        const float q1 = t2 * e1x - t0 * e1z;
        const float q2 = t0 * e1y - t1 * e1x;
        const float w = (v[0] * q0 + v[1] * q1 + v[2] * q2) * inv;
        if (w < -err || u + w > 1.0f + 2.0f * err) continue;
        const float t = (e2x * q0 + e2y * q1 + e2z * q2) * inv;
        // time error: relative err plus the position-scale term
        const float tErr = err * (fabsf(t) + (fabsf(t0) + fabsf(t1) + fabsf(t2)) / fmaxf(vnorm, 1e-30f));
        if (t < -tErr) continue;                       // certain miss (behind)
        // on the entry face: |t| <= posTol/|v.n| <= posTol*|e1||e2|/|det|
        if (face == entryFace && t <= 2.0f * posTol * e12 * fabsf(inv)) continue;
        const bool inside = (u > err) && (u < 1.0f - err) && (w > err) && (u + w < 1.0f - 2.0f * err);
        if (!inside || t <= fmaxf(tErr, 1e-13f)) {
            h.ambiguous = true;
            continue;
        }
        if (t < h.t) {
            second = h.t; secondErr = h.terr;
            h.t = t; h.terr = tErr; h.face = face; h.tri = tag;
        } else if (t < second) {
            second = t; secondErr = tErr;
        }
    }
    if (h.face != -2 && second < FLT_MAX && second - h.t <= h.terr + secondErr) h.ambiguous = true;
    return h;
}

// ---------------------------------------------------------------------------
// Plane-based exit search for cells that are convex with planar faces.
//
// The exit of a ray from inside a convex cell is the face plane it reaches
// first among those it moves towards: t_f = (d_f - n_f.x) / (v.n_f) for
// v.n_f > 0. That takes one dot-product pair per face instead of a full
// triangle test per triangle. The result is only trusted when it is clear of
// every tie the triangle tests could resolve differently: a second plane
// reached within the error bound (edge or vertex), a tiny or negative t, a
// plane grazed while the particle sits on it, a position outside a face
// plane, and for quads a hit point within the bound of the split diagonal
// (which sub-triangle). Otherwise `ambiguous` is set and the caller runs the
// triangle search. The entry face (crossf) is never the exit: the particle
// sits on it and moves away from it.
// ---------------------------------------------------------------------------
template <typename Real>
struct PlaneHit {
    int face;
    int tri;       // -1 triangle face, 1/2 quad half
    int triIdx;    // index of that triangle in the cell's triangle list
    Real t;
    Real terr;
    bool ambiguous;
    int nb;        // the record's crossing: the cell on the other side, kNbLost or -(role + 1)
    float4 delta;  // FP32 path: the record's centre shift
};

template <typename Real>
__device__ __forceinline__ PlaneHit<Real> find_exit_planes(const DevMesh& M, int cell, int crossf, const Real x[3],
                                                           const Real v[3])
{
    constexpr Real eps = (sizeof(Real) == 8) ? (Real)1.1102230246251565e-16 : (Real)5.9604645e-8f;
    constexpr Real K = (sizeof(Real) == 8) ? (Real)64 : (Real)32;
    PlaneHit<Real> h{-2, -1, -1, (Real)0, (Real)0, false, 0, make_float4(0.f, 0.f, 0.f, 0.f)};
    const Real vnorm = fabs(v[0]) + fabs(v[1]) + fabs(v[2]);
    const Real xnorm = fabs(x[0]) + fabs(x[1]) + fabs(x[2]);
    Real best = (sizeof(Real) == 8) ? (Real)DBL_MAX : (Real)FLT_MAX;
    Real second = best, bestErr = 0, secondErr = 0;
    int bi = -1;
    bool amb = false;
    float4 bestDelta = make_float4(0.f, 0.f, 0.f, 0.f);
    const int b = M.faceStride ? cell * M.faceStride : M.faceOff[cell];
    const int e = M.faceStride ? b + M.faceStride : M.faceOff[cell + 1];
    for (int k = b; k < e; ++k) {
        const int4 rec = M.faceRec[k];
        float4 dk = make_float4(0.f, 0.f, 0.f, 0.f);
        if constexpr (sizeof(Real) == 4) dk = M.nbDeltaF[k];
        if (rec.x == crossf) continue;
        Real nx, ny, nz, d;
        if constexpr (sizeof(Real) == 8) {
            const double* pd = M.planeD + (size_t)k * 8;
            nx = pd[0]; ny = pd[1]; nz = pd[2]; d = pd[3];
        } else {
            const float4 pl = M.planeF[k];
            nx = pl.x; ny = pl.y; nz = pl.z; d = pl.w;
        }
        const Real vn = v[0] * nx + v[1] * ny + v[2] * nz;
        const Real num = d - (x[0] * nx + x[1] * ny + x[2] * nz);
        const Real dErr = K * eps * (fabs(d) + xnorm);
        const Real vErr = K * eps * vnorm;
        if (num < -dErr) amb = true;                    // outside this face plane
        if (vn <= vErr) {
            if (vn > -vErr && num <= dErr) amb = true;  // grazing the plane it sits on
            continue;
        }
        const Real t = num / vn;
        const Real tErr = (dErr + fabs(t) * vErr) / vn;
        if (t < best) {
            second = best; secondErr = bestErr;
            best = t; bestErr = tErr; bi = k;
            bestDelta = dk;
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
    h.terr = bestErr;
    h.tri = -1;
    h.triIdx = rec.y;
    h.nb = rec.w;
    h.delta = bestDelta;
    if (rec.z == 4) {
        Real mx, my, mz, md;
        if constexpr (sizeof(Real) == 8) {
            const double* pd = M.planeD + (size_t)bi * 8;
            mx = pd[4]; my = pd[5]; mz = pd[6]; md = pd[7];
        } else {
            const float4 dg = M.diagF[bi];
            mx = dg.x; my = dg.y; mz = dg.z; md = dg.w;
        }
        const Real px = x[0] + v[0] * best, py = x[1] + v[1] * best, pz = x[2] + v[2] * best;
        const Real side = mx * px + my * py + mz * pz - md;
        const Real sErr = K * eps * (fabs(md) + fabs(px) + fabs(py) + fabs(pz)) + vnorm * bestErr;
        if (fabs(side) <= sErr) amb = true;
        h.tri = side > (Real)0 ? 1 : 2;
        h.triIdx = rec.y + (h.tri == 2 ? 1 : 0);
    }
    h.ambiguous = amb;
    return h;
}

// ---------------------------------------------------------------------------
// Particle state in registers and the tracing loop.
// ---------------------------------------------------------------------------
template <typename Real>
struct PRegs {
    Real x[3];   // FP64: absolute; FP32: relative to the centre of `cell`
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
template <typename Real>
__device__ __forceinline__ void diffuse_reflect(const DevMesh& M, const DevConsts& C, int wslot, int tag,
                                                PRegs<Real>& p, Stream& rng)
{
    const int which = (tag == 2) ? 1 : 0;
    const Real r1 = rng.uniform<Real>();
    const Real r2 = rng.uniform<Real>();
    const Real al = rng.uniform<Real>();
    const Real r3 = rng.uniform<Real>();
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

// x += v t (scalar_product, src/ProcessDSMC.cpp:1611-1617)
template <typename Real>
__device__ __forceinline__ void advance(PRegs<Real>& p, Real t)
{
    if constexpr (sizeof(Real) == 8) {
        for (int d = 0; d < 3; ++d) p.x[d] = da(p.x[d], dm(p.v[d], t));
    } else {
        for (int d = 0; d < 3; ++d) p.x[d] += p.v[d] * t;
    }
}

// The tracing loop's state between two exit searches.
struct TraceState {
    int ifout;        // outcome so far
    int iter;         // exit searches made
    int crossf, tag;  // the face / triangle the particle entered through
    int entryFace;    // the face the particle sits on (mixed path)
    bool afterNone;   // the last hit had no handler: use the triangle search
    __device__ __forceinline__ void begin(int crossf0, int tag0)
    {
        ifout = kTraceStay;
        iter = 0;
        crossf = crossf0;
        tag = tag0;
        entryFace = crossf0;
        afterNone = false;
    }
};

// One pass of the tracing loop (traceParticleDtleft, src/ProcessDSMC.cpp:
// 149-221): an exit search from `cell` and either the advance to the end of
// the step or the crossing with its boundary handling. Returns true when the
// trace is over, with the outcome in st.ifout.
template <typename Real>
__device__ __forceinline__ bool trace_step(const DevMesh& M, const DevConsts& C, PRegs<Real>& p, int& cell,
                                           Real& dtleft, TraceState& st, Stream& rng, int istep,
                                           double* wallTally, TraceCounts& cnt, bool stopAtWall, TraceLog* log)
{
    int& ifout = st.ifout;
    int& crossf = st.crossf;
    int& tag = st.tag;
    int& entryFace = st.entryFace;
    bool& afterNone = st.afterNone;
    if (!(dtleft > (Real)0)) return true;
    {
        if (st.iter++ >= C.maxCross) { cnt.lost++; dtleft = 0; ifout = kTraceLost; return true; }
        int face, tri;
        Real t;
        bool stays;
        // a face chosen by the plane search comes with its record's crossing
        bool hint = false;
        int hintNb = 0;
        float4 hintDelta = make_float4(0.f, 0.f, 0.f, 0.f);
        if constexpr (sizeof(Real) == 8) {
            bool decided = false;
            if ((M.allConvex || M.convex[cell]) && !afterNone) {
                // plane decision, then the reference's exact test on that one
                // triangle for the bit-exact t; any doubt runs the full search
                const PlaneHit<double> ph = find_exit_planes<double>(M, cell, crossf, p.x, p.v);
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
            }
            hint = decided;
            if (!decided) {
                const ExitHit h = find_exit_exact(M, cell, crossf, tag, p.x, p.v);
                if (h.face == -2 || !isfinite(h.t) || h.t <= 0.0) { cnt.dropped++; dtleft = 0; ifout = kTraceDropped; return true; }
                face = h.face; tri = h.tri; t = h.t;
            }
            stays = t >= dtleft;
        } else {
            const float vnorm = sqrtf(p.v[0] * p.v[0] + p.v[1] * p.v[1] + p.v[2] * p.v[2]);
            // absolute uncertainty of the FP32 cell-relative position
            const float posTol = 64.0f * 5.9604645e-8f * (fabsf(p.x[0]) + fabsf(p.x[1]) + fabsf(p.x[2]));
            ExitHitF h;
            bool planes = false;
            if ((M.allConvex || M.convex[cell]) && !afterNone) {
                const PlaneHit<float> ph = find_exit_planes<float>(M, cell, crossf, p.x, p.v);
                h = ExitHitF{ph.face, ph.tri, ph.t, ph.terr, ph.ambiguous};
                planes = true;
                hintNb = ph.nb;
                hintDelta = ph.delta;
            } else {
                h = find_exit_f32(M, cell, crossf, tag, p.x, p.v, vnorm, entryFace, posTol);
            }
            bool amb = h.ambiguous;
            if (!amb && h.face != -2 &&
                fabsf(h.t - dtleft) <= h.terr + 4.8e-7f * (dtleft + (float)C.dtime)) amb = true;
            if (amb) {
                // Repeat this crossing step in exact FP64 from the same state.
                cnt.fallback++;
                const double* cc = M.cellCenter + (size_t)cell * 3;
                double xa[3] = {cc[0] + (double)p.x[0], cc[1] + (double)p.x[1], cc[2] + (double)p.x[2]};
                const double va[3] = {(double)p.v[0], (double)p.v[1], (double)p.v[2]};
                const ExitHit he = find_exit_exact(M, cell, crossf, tag, xa, va, entryFace, (double)posTol);
                if (he.face == -2 || !isfinite(he.t) || he.t <= 0.0) { cnt.dropped++; dtleft = 0; ifout = kTraceDropped; return true; }
                face = he.face; tri = he.tri;
                const double dl = (double)dtleft;
                if (he.t >= dl) {
                    for (int d = 0; d < 3; ++d) p.x[d] = (float)(da(xa[d], dm(va[d], dl)) - cc[d]);
                    dtleft = 0;
                    return true;
                }
                stays = false;
                t = (float)he.t;
                if (!(t < dtleft)) t = nextafterf(dtleft, 0.0f);
            } else {
                if (h.face == -2 || !(h.t > 0.0f)) { cnt.dropped++; dtleft = 0; ifout = kTraceDropped; return true; }
                face = h.face; tri = h.tri; t = h.t;
                stays = t >= dtleft;
                hint = planes;
            }
        }
        if (stays) {
            advance(p, dtleft);
            dtleft = 0;
            return true;
        }
        crossf = face;
        tag = tri;
        const int role = !hint ? (int)M.faceRole[face] : (hintNb >= 0 || hintNb == kNbLost) ? kRoleInterface : -(hintNb + 1);
        if (log && role != kRoleInterface && log->hitFace < 0) {
            log->hitFace = face;
            log->hitTri = tri;
            if (stopAtWall && role == kRoleWall) {
                advance(p, t);
                if constexpr (sizeof(Real) == 8) dtleft = ds(dtleft, t); else dtleft -= t;
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
            if constexpr (sizeof(Real) == 8) dtleft = ds(dtleft, t); else dtleft -= t;
            int next;
            int2 cc = make_int2(0, 0);
            if (hint) {
                next = hintNb;
            } else {
                cc = M.faceCells[face];
                if (cell == cc.x) next = cc.y;
                else if (cell == cc.y) next = cc.x;
                else next = cc.x;
            }
            if (next < 0 || next >= M.ncell) { cnt.lost++; dtleft = 0; ifout = kTraceLost; return true; }
            if constexpr (sizeof(Real) == 4) {
                if (hint) {
                    p.x[0] += hintDelta.x; p.x[1] += hintDelta.y; p.x[2] += hintDelta.z;
                } else {
                    const float4 dl = M.faceDelta[face];
                    const float sg = (cell == cc.x) ? 1.0f : -1.0f;
                    p.x[0] += sg * dl.x; p.x[1] += sg * dl.y; p.x[2] += sg * dl.z;
                }
            }
            cell = next;
            entryFace = face;
        } else if (role == kRoleInlet || role == kRoleOutlet) {
            cnt.removed++;
            dtleft = 0;
            ifout = kTraceRemoved; return true;
        } else if (role == kRoleWall) {
            if constexpr (sizeof(Real) == 8) dtleft = ds(dtleft, t); else dtleft -= t;
            const int ws = M.faceWall[face];
            const Real v0 = p.v[0], v1 = p.v[1], v2 = p.v[2], ir0 = p.ir;
            diffuse_reflect<Real>(M, C, ws, tri, p, rng);
            cnt.wall++;
            entryFace = face;
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
            if constexpr (sizeof(Real) == 8) dtleft = ds(dtleft, t); else dtleft -= t;
            specular_reflect<Real>(M, M.faceWall[face], tri, p);
            cnt.wall++;
            entryFace = face;
        }
        // kRoleNone: no handler (src/ProcessDSMC.cpp:1826-1827); the next
        // search excludes this face and the particle is dropped.
        afterNone = (role == kRoleNone);
    }
    return false;
}

// Trace one particle, starting in `cell` having entered through face
// `crossf` / triangle `tag` (-1/-1 for a particle at rest in its cell), for
// `dtleft` (updated: the time not flown when the trace stops). Returns the
// reference's outcome and leaves the final cell in `cell`.
template <typename Real>
__device__ int trace_particle(const DevMesh& M, const DevConsts& C, PRegs<Real>& p, int& cell,
                             int crossf, int tag, Real& dtleft, Stream& rng, int istep,
                             double* wallTally, TraceCounts& cnt, bool stopAtWall, TraceLog* log)
{
    TraceState st;
    st.begin(crossf, tag);
    while (!trace_step<Real>(M, C, p, cell, dtleft, st, rng, istep, wallTally, cnt, stopAtWall, log)) {
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
