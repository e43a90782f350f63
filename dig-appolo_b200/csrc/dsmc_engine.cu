// Host engine behind the C ABI (include/dsmc_gpu.h): builds the device mesh
// caches from the reference's mesh arrays, owns all device state of one
// case, and orchestrates the step stages on one stream (replayed as a CUDA
// graph in production).
#include "dsmc_gpu.h"
#include "dsmc_meshio.h"
#include "dsmc_kernels.cuh"
#include "dsmc_hostpack.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <numeric>
#include <stdexcept>
#include <string>
#include <vector>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

namespace dsmc {

static_assert(sizeof(DsmcCellRec) == 120, "DsmcCell layout");
static_assert(sizeof(DsmcEdgeRec) == 88, "DsmcEdge layout");
static_assert(sizeof(DsmcMeshMessage) == 344, "meshMessage layout");

namespace {

constexpr unsigned char kSplit02 = 0;
constexpr unsigned char kSplit13 = 1;

// meshImport::decode_quad_split_tag, src/meshImport.h:309-327
void decode_split(unsigned char tag, int t0[3], int t1[3])
{
    if (tag == kSplit02) {
        t0[0] = 0; t0[1] = 1; t0[2] = 2; t1[0] = 0; t1[1] = 2; t1[2] = 3;
    } else if (tag == kSplit13) {
        t0[0] = 0; t0[1] = 1; t0[2] = 3; t1[0] = 1; t1[1] = 2; t1[2] = 3;
    } else {
        t0[0] = t0[1] = t0[2] = -1; t1[0] = t1[1] = t1[2] = -1;
    }
}

// ProcessDSMC::normalize, src/ProcessDSMC.cpp:1564-1570
void normalize3(double v[3])
{
    const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= len;
    v[1] /= len;
    v[2] /= len;
}

// MeshparticalInitial::crossProduct, src/MeshparticalInitial.cpp:819-823
void cross3(const double* a, const double* b, double* r)
{
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}

// MeshparticalInitial::dotProduct, src/MeshparticalInitial.cpp:829-835
double dot3(const double* a, const double* b)
{
    double r = 0.0;
    for (int i = 0; i < 3; ++i) r += a[i] * b[i];
    return r;
}

// ProcessDSMC::buildRotationMatrix, src/ProcessDSMC.cpp:1583-1603
void rotation(const double* n, double R[9])
{
    double t1[3], t2[3];
    if ((std::fabs(n[0]) <= std::fabs(n[1])) && (std::fabs(n[0]) <= std::fabs(n[2]))) {
        t1[0] = 0.0; t1[1] = n[2]; t1[2] = -n[1];
    } else if (std::fabs(n[1]) < std::fabs(n[2])) {
        t1[0] = n[2]; t1[1] = 0.0; t1[2] = -n[0];
    } else {
        t1[0] = n[1]; t1[1] = -n[0]; t1[2] = 0.0;
    }
    normalize3(t1);
    cross3(n, t1, t2);
    normalize3(t2);
    R[0] = t1[0]; R[1] = t2[0]; R[2] = n[0];
    R[3] = t1[1]; R[4] = t2[1]; R[5] = n[1];
    R[6] = t1[2]; R[7] = t2[2]; R[8] = n[2];
}

template <typename T>
struct DevArray {
    T* p = nullptr;
    size_t n = 0;
};

}  // namespace

struct Engine {
    int device = 0;
    int smCount = 148;
    cudaStream_t stream = nullptr;
    int precision = DSMC_PRECISION_FP64;
    DsmcCaseParams params{};
    DsmcMeshMessage mess{};
    int ncell = 0, nface = 0, npoint = 0, ntri = 0, nwall = 0, nconvex = 0;
    std::vector<DsmcCellRec> cells;
    std::vector<DsmcEdgeRec> edges;
    std::vector<double> points;
    std::vector<unsigned char> split;
    std::vector<int> faceRole;
    std::vector<int> faceWallHost;
    std::vector<double> cellCenterHost;
    std::string err;

    // device allocations
    std::vector<void*> allocs;
    DevMesh M{};
    DevConsts C{};
    DevPatches P{};
    void* buf[2][8] = {};          // x,y,z,vx,vy,vz,ir (Real), cell (int)
    int* start[2] = {nullptr, nullptr};
    int* rank = nullptr;
    int* idx = nullptr;
    int* countSlot = nullptr;
    int* scanPartial = nullptr;
    double* crmax = nullptr;
    double* remColl = nullptr;
    double* remInj = nullptr;
    double* acc = nullptr;
    double* record = nullptr;
    double* local = nullptr;
    double* finalRecord = nullptr;
    double* stepMom = nullptr;
    unsigned char* sparseState = nullptr;
    int* sparseAccum = nullptr;
    double* windowSamples = nullptr;
    char* windowValid = nullptr;
    double* wallTally = nullptr;
    StepCtl* ctl = nullptr;
    unsigned long long* counters = nullptr;
    int* cellList = nullptr;
    int4* cellItem = nullptr;
    double2* cellItemC = nullptr;
    int* cellWork = nullptr;
    int* cellPairs = nullptr;
    double* cellCons = nullptr;
    int* errorWord = nullptr;
    int* uploadFlag = nullptr;     // upload_check_kernel's flags
    int* placeFirst = nullptr;     // [nplace] cell-local first particle of each placement tetrahedron (fill)
    // GSIS particle update (allocated on first use)
    double* gsisNs = nullptr;
    unsigned char* gsisAcc = nullptr;
    int* gsisFlag = nullptr;
    unsigned long long* gsisTally = nullptr;
    uint32_t gsisEpoch = 0;

    int64_t capacity = 0;
    int cur = 0;                   // which buffer holds the particles
    bool haveParticles = false;
    bool pendingInject = false;    // injected particles not yet sorted
    bool localLazy = false;
    int lastIstep = 0;             // step of the last statistic_macro
    int curIstep = 0;              // step of the last stage call
    uint64_t steps = 0;
    int hostNLive = 0;

    cudaGraphExec_t graph[2] = {nullptr, nullptr};
    LaunchShape shape;             // launch shapes (dsmc_set_launch_shape, dsmc_autotune)
    int generation = 0;            // bumped whenever captured graphs become stale
    bool devIstepValid = false;    // ctl->istep on the device equals curIstep
    bool timing = false;
    cudaEvent_t ev[6] = {};
    double stageMs[5] = {0, 0, 0, 0, 0};
    int64_t timedSteps = 0;
    // pinned host chunks that pageable upload arrays pass through (allocated
    // on the first such upload), and the events of their last copies
    static constexpr size_t kHostStage = size_t(64) << 20;
    void* hostStage[2] = {nullptr, nullptr};
    cudaEvent_t stageEv[2] = {nullptr, nullptr};

    ~Engine() { release(); }

    void release()
    {
        if (device >= 0) cudaSetDevice(device);
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        for (auto& e : ev)
            if (e) { cudaEventDestroy(e); e = nullptr; }
        for (int b = 0; b < 2; ++b) {
            if (stageEv[b]) { cudaEventDestroy(stageEv[b]); stageEv[b] = nullptr; }
            if (hostStage[b]) { cudaFreeHost(hostStage[b]); hostStage[b] = nullptr; }
        }
        for (void* p : allocs) cudaFree(p);
        allocs.clear();
        if (stream) { cudaStreamDestroy(stream); stream = nullptr; }
    }

    bool fail(const std::string& m)
    {
        err = m;
        return false;
    }
    bool cuda(cudaError_t e, const char* what)
    {
        if (e == cudaSuccess) return true;
        err = std::string(what) + ": " + cudaGetErrorString(e);
        return false;
    }
    template <typename T>
    bool alloc(T*& p, size_t n, bool zero = true)
    {
        void* q = nullptr;
        const size_t bytes = std::max<size_t>(n, 1) * sizeof(T);
        const cudaError_t e = cudaMalloc(&q, bytes);
        if (e != cudaSuccess) {
            err = std::string("cudaMalloc ") + std::to_string(bytes) + " B: " + cudaGetErrorString(e);
            return false;
        }
        allocs.push_back(q);
        p = static_cast<T*>(q);
        if (zero) return cuda(cudaMemsetAsync(q, 0, bytes, stream), "cudaMemset");
        return true;
    }
    template <typename T>
    bool upload(T*& p, const std::vector<T>& h)
    {
        if (!alloc(p, h.size(), false)) return false;
        if (h.empty()) return true;
        return cuda(cudaMemcpyAsync(p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice, stream), "upload");
    }
    void freePtr(void* p)
    {
        if (!p) return;
        cudaFree(p);
        allocs.erase(std::remove(allocs.begin(), allocs.end(), p), allocs.end());
    }

    size_t realSize() const { return precision == DSMC_PRECISION_MIXED ? sizeof(float) : sizeof(double); }

    int roleOfTag(int tag, bool* inject) const
    {
        for (int z = 0; z < params.nzones && z < DSMC_MAX_ZONES; ++z)
            if (params.zone_tag[z] == tag) {
                if (inject) *inject = params.zone_inject[z] != 0;
                return params.zone_role[z];
            }
        if (inject) *inject = false;
        return DSMC_ROLE_NONE;
    }

    bool loadPoint(int idx, double P3[3]) const
    {
        if (idx < 0 || (size_t)idx * 3 + 2 >= points.size()) return false;
        P3[0] = points[(size_t)idx * 3];
        P3[1] = points[(size_t)idx * 3 + 1];
        P3[2] = points[(size_t)idx * 3 + 2];
        return true;
    }

    // ------------------------------------------------------------------
    // Placement tetrahedra of every cell, as buildCellInitTets
    // (src/MeshparticalInitial.cpp:172-355, src/ProcessGSIS.cpp:748-964):
    // a cell with 4 distinct nodes is its own tetrahedron (nodes in order of
    // first appearance over its faces); a cell with 5 nodes and one quad is
    // split into the two base triangles (the quad's split tag) with the apex;
    // any other cell into its centre with each face triangle. A tetrahedron
    // of zero or non-finite volume rejects that decomposition; a cell that
    // none fits gets no tetrahedra (the fill places nothing there and GSIS
    // copies go to the cell centre).
    std::vector<int> placeOffHost;
    std::vector<double> placeVolHost;

    void buildPlacement(std::vector<double>& V)
    {
        placeOffHost.assign((size_t)ncell + 1, 0);
        placeVolHost.clear();
        V.clear();
        // tetAbsVolume / appendCenterFaceTet, src/ProcessGSIS.cpp:660-675, 829-870
        auto tetVol = [](const double* P0, const double* P1, const double* P2, const double* P3) {
            const double ax = P1[0] - P0[0], ay = P1[1] - P0[1], az = P1[2] - P0[2];
            const double bx = P2[0] - P0[0], by = P2[1] - P0[1], bz = P2[2] - P0[2];
            const double cx = P3[0] - P0[0], cy = P3[1] - P0[1], cz = P3[2] - P0[2];
            const double crx = by * cz - bz * cy;
            const double cry = bz * cx - bx * cz;
            const double crz = bx * cy - by * cx;
            return std::fabs(ax * crx + ay * cry + az * crz) / 6.0;
        };
        struct Tet { double v[12]; double vol; };
        std::vector<Tet> tets;
        auto vertexTet = [&](int n0, int n1, int n2, int n3) {
            Tet t;
            const int n[4] = {n0, n1, n2, n3};
            for (int k = 0; k < 4; ++k)
                if (!loadPoint(n[k], &t.v[3 * k])) return false;
            t.vol = tetVol(&t.v[0], &t.v[3], &t.v[6], &t.v[9]);
            if (!(t.vol > 0.0) || !std::isfinite(t.vol)) return false;
            tets.push_back(t);
            return true;
        };
        auto centerTet = [&](int c, int n0, int n1, int n2) {
            Tet t;
            for (int d = 0; d < 3; ++d) t.v[d] = cellCenterHost[(size_t)c * 3 + d];
            const int n[3] = {n0, n1, n2};
            for (int k = 0; k < 3; ++k)
                if (!loadPoint(n[k], &t.v[3 + 3 * k])) return false;
            t.vol = tetVol(&t.v[0], &t.v[3], &t.v[6], &t.v[9]);
            if (!(t.vol > 0.0) || !std::isfinite(t.vol)) return false;
            tets.push_back(t);
            return true;
        };
        auto validFace = [&](int f) { return f >= 0 && f < nface; };
        std::vector<int> uniq;
        for (int c = 0; c < ncell; ++c) {
            placeOffHost[(size_t)c] = (int)placeVolHost.size();
            const DsmcCellRec& cl = cells[(size_t)c];
            const int nf = std::min(cl.num, 6);
            // collectCellUniqueNodes
            bool nodesOk = true;
            uniq.clear();
            for (int m = 0; m < nf && nodesOk; ++m) {
                const int f = cl.cell2face[m];
                if (!validFace(f)) { nodesOk = false; break; }
                const DsmcEdgeRec& e = edges[(size_t)f];
                if (e.faceType != 3 && e.faceType != 4) { nodesOk = false; break; }
                for (int k = 0; k < e.faceType; ++k) {
                    const int node = e.faceMap[k];
                    if (node < 0 || (size_t)node * 3 + 2 >= points.size()) { nodesOk = false; break; }
                    if (std::find(uniq.begin(), uniq.end(), node) == uniq.end()) uniq.push_back(node);
                }
            }
            tets.clear();
            bool done = false;
            // appendTetCellTets
            if (nodesOk && uniq.size() == 4u) done = vertexTet(uniq[0], uniq[1], uniq[2], uniq[3]);
            // appendPyramidCellTets
            if (!done) {
                tets.clear();
                int quad = -1;
                bool ok = true;
                for (int m = 0; m < nf; ++m) {
                    const int f = cl.cell2face[m];
                    if (!validFace(f)) { ok = false; break; }
                    if (edges[(size_t)f].faceType == 4) {
                        if (quad >= 0) { ok = false; break; }
                        quad = f;
                    }
                }
                if (ok && quad >= 0 && nodesOk && uniq.size() == 5u) {
                    const DsmcEdgeRec& base = edges[(size_t)quad];
                    int apex = -1;
                    for (int node : uniq) {
                        bool onBase = false;
                        for (int k = 0; k < 4; ++k) onBase = onBase || base.faceMap[k] == node;
                        if (!onBase) { apex = node; break; }
                    }
                    if (apex >= 0) {
                        int t0[3], t1[3];
                        decode_split(split[(size_t)quad], t0, t1);
                        if (t0[0] < 0 || t1[0] < 0) decode_split(kSplit02, t0, t1);
                        done = vertexTet(base.faceMap[t0[0]], base.faceMap[t0[1]], base.faceMap[t0[2]], apex) &&
                               vertexTet(base.faceMap[t1[0]], base.faceMap[t1[1]], base.faceMap[t1[2]], apex);
                    }
                }
            }
            // appendCenterFaceTets
            if (!done) {
                tets.clear();
                bool ok = true;
                for (int m = 0; m < nf && ok; ++m) {
                    const int f = cl.cell2face[m];
                    if (!validFace(f)) { ok = false; break; }
                    const DsmcEdgeRec& e = edges[(size_t)f];
                    if (e.faceType == 3) {
                        ok = centerTet(c, e.faceMap[0], e.faceMap[1], e.faceMap[2]);
                    } else if (e.faceType == 4) {
                        int t0[3], t1[3];
                        decode_split(split[(size_t)f], t0, t1);
                        if (t0[0] < 0 || t1[0] < 0) decode_split(kSplit02, t0, t1);
                        ok = centerTet(c, e.faceMap[t0[0]], e.faceMap[t0[1]], e.faceMap[t0[2]]) &&
                             centerTet(c, e.faceMap[t1[0]], e.faceMap[t1[1]], e.faceMap[t1[2]]);
                    } else {
                        ok = false;
                    }
                }
                done = ok && !tets.empty();
            }
            if (!done) continue;
            for (const Tet& t : tets) {
                V.insert(V.end(), t.v, t.v + 12);
                placeVolHost.push_back(t.vol);
            }
        }
        placeOffHost[(size_t)ncell] = (int)placeVolHost.size();
    }

    // ------------------------------------------------------------------
    bool build(const DsmcMeshDesc* md, const DsmcMeshMessage* mm, const DsmcCaseParams* pp, int dev)
    {
        if (!md || !mm || !pp) return fail("null argument");
        if (md->ncell <= 0 || md->nface <= 0 || md->npoint <= 0 || !md->cells || !md->edges || !md->localPointXY)
            return fail("empty or incomplete mesh");
        params = *pp;
        mess = *mm;
        precision = params.precision;
        if (precision != DSMC_PRECISION_FP64 && precision != DSMC_PRECISION_MIXED) return fail("bad precision");
        if (params.nevery <= 0 || params.nrepeat <= 0 || params.nscheme <= 0) return fail("bad sampling controls");
        if (params.nzones < 0 || params.nzones > DSMC_MAX_ZONES) return fail("nzones outside [0, DSMC_MAX_ZONES]");
        for (int z = 0; z < params.nzones; ++z)
            if (params.zone_role[z] < DSMC_ROLE_NONE || params.zone_role[z] > DSMC_ROLE_SPECULAR)
                return fail("unknown zone role");
        if (params.max_crossings <= 0) params.max_crossings = 4096;
        if (!(mess.dtime > 0.0) || !(mess.Neff > 0.0) || !(mess.v_rms > 0.0)) return fail("bad mesh message");
        if (dev >= 0) {
            if (!cuda(cudaSetDevice(dev), "cudaSetDevice")) return false;
            device = dev;
        } else if (!cuda(cudaGetDevice(&device), "cudaGetDevice")) {
            return false;
        }
        cudaDeviceGetAttribute(&smCount, cudaDevAttrMultiProcessorCount, device);
        shape.smCount = smCount;
        if (!cuda(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking), "cudaStreamCreate")) return false;
        ncell = md->ncell;
        nface = md->nface;
        npoint = md->npoint;
        cells.assign(md->cells, md->cells + ncell);
        edges.assign(md->edges, md->edges + nface);
        points.assign(md->localPointXY, md->localPointXY + (size_t)npoint * 3);
        split.assign((size_t)nface, 255);
        if (md->faceSplitTag) split.assign(md->faceSplitTag, md->faceSplitTag + nface);

        cellCenterHost.resize((size_t)ncell * 3);
        for (int c = 0; c < ncell; ++c)
            for (int d = 0; d < 3; ++d) cellCenterHost[(size_t)c * 3 + d] = cells[(size_t)c].cellXY[d];

        // --- face roles (BoundaryConditionTable::byTag) -------------------------------
        faceRole.assign((size_t)nface, DSMC_ROLE_NONE);
        for (int f = 0; f < nface; ++f) faceRole[(size_t)f] = roleOfTag(edges[(size_t)f].faceTag, nullptr);

        // --- triangle cache: rebuildFaceTraversalCache, src/ProcessDSMCGeometry.cpp:145-214
        std::vector<int> triOffset((size_t)ncell + 1, 0);
        std::vector<double> triD;
        std::vector<int2> triFT;
        triD.reserve((size_t)ncell * 8 * 9);
        for (int lc = 0; lc < ncell; ++lc) {
            triOffset[(size_t)lc] = (int)triFT.size();
            const DsmcCellRec& cl = cells[(size_t)lc];
            const double* cc = &cellCenterHost[(size_t)lc * 3];
            auto appendTri = [&](int faceid, int tag, int ia, int ib, int ic) {
                double A[3], B[3], Cc[3];
                if (!loadPoint(ia, A) || !loadPoint(ib, B) || !loadPoint(ic, Cc)) return;
                const double e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
                const double e2[3] = {Cc[0] - A[0], Cc[1] - A[1], Cc[2] - A[2]};
                for (int d = 0; d < 3; ++d) triD.push_back(A[d]);
                for (int d = 0; d < 3; ++d) triD.push_back(e1[d]);
                for (int d = 0; d < 3; ++d) triD.push_back(e2[d]);
                triFT.push_back(make_int2(faceid, tag));
            };
            for (int m = 0; m < cl.num && m < 6; ++m) {
                const int faceid = cl.cell2face[m];
                if (faceid < 0 || faceid >= nface) continue;
                const DsmcEdgeRec& face = edges[(size_t)faceid];
                const int* ids = face.faceMap;
                if (face.faceType == 3) {
                    appendTri(faceid, -1, ids[0], ids[1], ids[2]);
                    continue;
                }
                if (face.faceType != 4) continue;
                int t0[3], t1[3];
                decode_split(split[(size_t)faceid], t0, t1);
                if (t0[0] < 0 || t1[0] < 0) decode_split(kSplit02, t0, t1);
                appendTri(faceid, 1, ids[t0[0]], ids[t0[1]], ids[t0[2]]);
                appendTri(faceid, 2, ids[t1[0]], ids[t1[1]], ids[t1[2]]);
            }
        }
        triOffset[(size_t)ncell] = (int)triFT.size();
        ntri = (int)triFT.size();

        // --- face planes for the plane-based exit search: per cell, its faces
        //     in cell2face order with outward unit normal and offset, the
        //     quad diagonal side test, and a flag for cells that are convex
        //     with planar faces (only those take the plane path)
        std::vector<int> faceOff((size_t)ncell + 1, 0);
        std::vector<int4> faceRec;
        std::vector<float4> planeF, diagF;
        std::vector<double> planeD;
        std::vector<unsigned char> convex((size_t)ncell, 0);
        for (int lc = 0; lc < ncell; ++lc) {
            faceOff[(size_t)lc] = (int)faceRec.size();
            const DsmcCellRec& cl = cells[(size_t)lc];
            const double* cc = &cellCenterHost[(size_t)lc * 3];
            bool ok = cl.num > 0 && cl.num <= 6;
            int triIdx = triOffset[(size_t)lc];
            std::vector<double> cellNodes;
            for (int m = 0; m < cl.num && m < 6 && ok; ++m) {
                const int f = cl.cell2face[m];
                if (f < 0 || f >= nface) { ok = false; break; }
                const DsmcEdgeRec& e = edges[(size_t)f];
                for (int q = 0; q < e.faceType && q < 4; ++q) {
                    double P3[3];
                    if (!loadPoint(e.faceMap[q], P3)) { ok = false; break; }
                    cellNodes.insert(cellNodes.end(), P3, P3 + 3);
                }
            }
            double Lc = 0.0;
            for (size_t q = 0; q + 2 < cellNodes.size(); q += 3)
                for (int d = 0; d < 3; ++d) Lc = std::max(Lc, std::fabs(cellNodes[q + d] - cc[d]));
            for (int m = 0; m < cl.num && m < 6 && ok; ++m) {
                const int f = cl.cell2face[m];
                const DsmcEdgeRec& e = edges[(size_t)f];
                const int type = e.faceType;
                if (type != 3 && type != 4) { ok = false; break; }
                double Pn[4][3];
                for (int q = 0; q < type; ++q) loadPoint(e.faceMap[q], Pn[q]);
                int t0[3] = {0, 1, 2}, t1[3] = {0, 2, 3};
                if (type == 4) {
                    decode_split(split[(size_t)f], t0, t1);
                    if (t0[0] < 0 || t1[0] < 0) decode_split(kSplit02, t0, t1);
                }
                const double* A = Pn[t0[0]];
                const double a1[3] = {Pn[t0[1]][0] - A[0], Pn[t0[1]][1] - A[1], Pn[t0[1]][2] - A[2]};
                const double a2[3] = {Pn[t0[2]][0] - A[0], Pn[t0[2]][1] - A[1], Pn[t0[2]][2] - A[2]};
                double n[3];
                cross3(a1, a2, n);
                const double nl = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
                if (!(nl > 0.0)) { ok = false; break; }
                for (int d = 0; d < 3; ++d) n[d] /= nl;
                double fc[3] = {0, 0, 0};
                for (int q = 0; q < type; ++q)
                    for (int d = 0; d < 3; ++d) fc[d] += Pn[q][d] / type;
                if ((fc[0] - cc[0]) * n[0] + (fc[1] - cc[1]) * n[1] + (fc[2] - cc[2]) * n[2] < 0.0)
                    for (double& x : n) x = -x;
                const double dAbs = n[0] * A[0] + n[1] * A[1] + n[2] * A[2];
                // planarity and convexity (every node of the cell on the inner side)
                const double tol = 1e-9 * std::max(Lc, 1e-300);
                for (int q = 0; q < type && ok; ++q)
                    if (std::fabs(n[0] * Pn[q][0] + n[1] * Pn[q][1] + n[2] * Pn[q][2] - dAbs) > tol) ok = false;
                for (size_t q = 0; q + 2 < cellNodes.size() && ok; q += 3)
                    if (n[0] * cellNodes[q] + n[1] * cellNodes[q + 1] + n[2] * cellNodes[q + 2] - dAbs > tol) ok = false;
                double mv[3] = {0, 0, 0}, md = 0.0;
                if (type == 4) {
                    // diagonal of the split and the in-plane normal to it,
                    // oriented so that the first triangle's side is positive
                    const int dA = t0[0] == t1[0] ? t0[0] : t1[0];   // split 02: 0; split 13: 1
                    const int dB = t0[0] == t1[0] ? t0[2] : t1[2];   // split 02: 2; split 13: 3
                    const double dv[3] = {Pn[dB][0] - Pn[dA][0], Pn[dB][1] - Pn[dA][1], Pn[dB][2] - Pn[dA][2]};
                    cross3(n, dv, mv);
                    const double ml = std::sqrt(mv[0] * mv[0] + mv[1] * mv[1] + mv[2] * mv[2]);
                    if (!(ml > 0.0)) { ok = false; break; }
                    for (double& x : mv) x /= ml;
                    int only0 = -1;   // a node of the first triangle off the diagonal
                    for (int q = 0; q < 3; ++q)
                        if (t0[q] != dA && t0[q] != dB) only0 = t0[q];
                    const double* Q = Pn[only0];
                    if (mv[0] * (Q[0] - Pn[dA][0]) + mv[1] * (Q[1] - Pn[dA][1]) + mv[2] * (Q[2] - Pn[dA][2]) < 0.0)
                        for (double& x : mv) x = -x;
                    md = mv[0] * Pn[dA][0] + mv[1] * Pn[dA][1] + mv[2] * Pn[dA][2];
                }
                faceRec.push_back(make_int4(f, triIdx, type, 0));
                triIdx += (type == 4) ? 2 : 1;
                const double dRel = n[0] * (A[0] - cc[0]) + n[1] * (A[1] - cc[1]) + n[2] * (A[2] - cc[2]);
                double mdRel = 0.0;
                if (type == 4) {
                    const double mcc = mv[0] * cc[0] + mv[1] * cc[1] + mv[2] * cc[2];
                    mdRel = md - mcc;
                }
                planeF.push_back(make_float4((float)n[0], (float)n[1], (float)n[2], (float)dRel));
                diagF.push_back(make_float4((float)mv[0], (float)mv[1], (float)mv[2], (float)mdRel));
                const double rec[8] = {n[0], n[1], n[2], dAbs, mv[0], mv[1], mv[2], md};
                planeD.insert(planeD.end(), rec, rec + 8);
            }
            if (ok && triIdx != triOffset[(size_t)lc + 1]) ok = false;
            if (!ok) {
                // the tri path serves this cell; drop any partial records
                faceRec.resize((size_t)faceOff[(size_t)lc]);
                planeF.resize((size_t)faceOff[(size_t)lc]);
                diagF.resize((size_t)faceOff[(size_t)lc]);
                planeD.resize((size_t)faceOff[(size_t)lc] * 8);
            }
            convex[(size_t)lc] = ok ? 1 : 0;
        }
        faceOff[(size_t)ncell] = (int)faceRec.size();
        nconvex = 0;
        for (unsigned char c : convex) nconvex += c;

        // --- wall / specular slots and rotations (getWallNormal +
        //     processFacesQuadNormals + buildRotationMatrix)
        auto quadNormals = [&](int fid, double n1[3], double n2[3]) -> bool {
            const DsmcEdgeRec& e = edges[(size_t)fid];
            double P4[4][3];
            for (int k = 0; k < 4; ++k)
                if (!loadPoint(e.faceMap[k], P4[k])) return false;
            unsigned char tag = split[(size_t)fid];
            int t0[3], t1[3];
            decode_split(tag, t0, t1);
            if (t0[0] < 0 || t1[0] < 0) decode_split(kSplit02, t0, t1);
            auto make = [&](const int tri[3], double n[3]) {
                const double* X = P4[tri[0]];
                const double* Y = P4[tri[1]];
                const double* Z = P4[tri[2]];
                const double e1[3] = {Y[0] - X[0], Y[1] - X[1], Y[2] - X[2]};
                const double e2[3] = {Z[0] - X[0], Z[1] - X[1], Z[2] - X[2]};
                cross3(e1, e2, n);
                normalize3(n);
                if (dot3(e.edgeNormal, n) < 0.0) {
                    n[0] *= -1.0; n[1] *= -1.0; n[2] *= -1.0;
                }
            };
            make(t0, n1);
            make(t1, n2);
            return true;
        };
        faceWallHost.assign((size_t)nface, -1);
        std::vector<double> wallRot;
        std::vector<float> wallRotF;
        for (int f = 0; f < nface; ++f) {
            const int role = faceRole[(size_t)f];
            if (role != DSMC_ROLE_WALL && role != DSMC_ROLE_SPECULAR) continue;
            faceWallHost[(size_t)f] = nwall++;
            const DsmcEdgeRec& e = edges[(size_t)f];
            double nbase[3] = {e.edgeNormal[0], e.edgeNormal[1], e.edgeNormal[2]};
            normalize3(nbase);
            double n1[3] = {nbase[0], nbase[1], nbase[2]}, n2[3] = {nbase[0], nbase[1], nbase[2]};
            if (e.faceType == 4) {
                double q1[3], q2[3];
                if (quadNormals(f, q1, q2)) {
                    std::memcpy(n1, q1, sizeof n1);
                    std::memcpy(n2, q2, sizeof n2);
                }
            }
            double R[9];
            rotation(n1, R);
            for (int k = 0; k < 9; ++k) { wallRot.push_back(R[k]); wallRotF.push_back((float)R[k]); }
            rotation(n2, R);
            for (int k = 0; k < 9; ++k) { wallRot.push_back(R[k]); wallRotF.push_back((float)R[k]); }
        }

        // --- face cells / deltas
        std::vector<int2> faceCells((size_t)nface);
        std::vector<unsigned char> roleU8((size_t)nface);
        for (int f = 0; f < nface; ++f) {
            const int c0 = edges[(size_t)f].faceMap[4], c1 = edges[(size_t)f].faceMap[5];
            faceCells[(size_t)f] = make_int2(c0, c1);
            roleU8[(size_t)f] = (unsigned char)faceRole[(size_t)f];
        }

        // --- what a crossing through each face record needs, kept with the
        //     record so the trace reads no per-face array: the cell on the
        //     other side (interface faces, as the trace picks it) or the
        //     face's role
        for (int lc = 0; lc < ncell; ++lc) {
            for (int k = faceOff[(size_t)lc]; k < faceOff[(size_t)lc + 1]; ++k) {
                const int f = faceRec[(size_t)k].x;
                const int role = faceRole[(size_t)f];
                int nb;
                if (role == DSMC_ROLE_INTERFACE) {
                    const int2 fc = faceCells[(size_t)f];
                    const int next = (lc == fc.x) ? fc.y : (lc == fc.y) ? fc.x : fc.x;
                    nb = (next >= 0 && next < ncell) ? next : kNbLost;
                } else {
                    nb = -(role + 1);
                }
                faceRec[(size_t)k].w = nb;
            }
        }

        // --- the mixed path's exit test (certain_exit_f32) per record: the
        //     smallest |e1 x e2| of the record's triangles (the reference's
        //     determinant is |v.n| times it), 0 when a triangle is so
        //     ill-conditioned (|e1||e2| / |e1 x e2| > 1024) that its FP64
        //     test could round far from the plane arithmetic; and the cell's
        //     length scale
        std::vector<float2> recAux(faceRec.size(), make_float2(0.0f, 0.0f));
        for (int lc = 0; lc < ncell; ++lc) {
            const double* cc = &cellCenterHost[(size_t)lc * 3];
            double lmax[3] = {0.0, 0.0, 0.0};
            for (int t = triOffset[(size_t)lc]; t < triOffset[(size_t)lc + 1]; ++t) {
                const double* T = &triD[(size_t)t * 9];
                const double P[3][3] = {{T[0], T[1], T[2]},
                                        {T[0] + T[3], T[1] + T[4], T[2] + T[5]},
                                        {T[0] + T[6], T[1] + T[7], T[2] + T[8]}};
                for (int q = 0; q < 3; ++q)
                    for (int d = 0; d < 3; ++d) lmax[d] = std::max(lmax[d], std::fabs(P[q][d] - cc[d]));
            }
            const float lscale = (float)((lmax[0] + lmax[1] + lmax[2]) * (1.0 + 1e-6));
            for (int k = faceOff[(size_t)lc]; k < faceOff[(size_t)lc + 1]; ++k) {
                const int4 rec = faceRec[(size_t)k];
                double detMin = DBL_MAX;
                for (int q = 0; q < (rec.z == 4 ? 2 : 1); ++q) {
                    const double* T = &triD[(size_t)(rec.y + q) * 9];
                    double cr[3];
                    cross3(T + 3, T + 6, cr);
                    const double a = std::sqrt(cr[0] * cr[0] + cr[1] * cr[1] + cr[2] * cr[2]);
                    const double l1 = std::sqrt(T[3] * T[3] + T[4] * T[4] + T[5] * T[5]);
                    const double l2 = std::sqrt(T[6] * T[6] + T[7] * T[7] + T[8] * T[8]);
                    const double m = (a > 0.0 && l1 * l2 <= 1024.0 * a) ? a : 0.0;
                    detMin = std::min(detMin, m);
                }
                // rounded down: the device bound must not exceed the true value
                const float df = (float)(detMin * (1.0 - 1e-6));
                recAux[(size_t)k] = make_float2(df, lscale);
            }
        }
        // every cell convex with the same number of faces: records at cell * F
        int faceStride = nconvex == ncell && ncell > 0 ? faceOff[1] - faceOff[0] : 0;
        for (int lc = 0; lc < ncell && faceStride; ++lc)
            if (faceOff[(size_t)lc] != lc * faceStride) faceStride = 0;

        // --- neighbour slots for the counting sort
        std::vector<int> c2c((size_t)ncell * 6, -1);
        std::vector<signed char> rev((size_t)ncell * 6, -1);
        std::vector<double> vol((size_t)ncell);
        for (int c = 0; c < ncell; ++c) {
            vol[(size_t)c] = cells[(size_t)c].area;
            for (int j = 0; j < 6 && j < cells[(size_t)c].num; ++j) c2c[(size_t)c * 6 + j] = cells[(size_t)c].cell2cell[j];
        }
        for (int c = 0; c < ncell; ++c) {
            for (int j = 0; j < 6 && j < cells[(size_t)c].num; ++j) {
                const int nb = c2c[(size_t)c * 6 + j];
                const int f = cells[(size_t)c].cell2face[j];
                if (nb < 0 || nb >= ncell) continue;
                for (int p = 0; p < 6 && p < cells[(size_t)nb].num; ++p)
                    if (cells[(size_t)nb].cell2face[p] == f) { rev[(size_t)c * 6 + j] = (signed char)p; break; }
            }
        }

        // --- inlet emit patches: rebuildBoundaryEmitCache, src/ProcessDSMC.cpp:583-768
        if (!buildPatches()) return false;

        // --- device constants
        C.dtime = mess.dtime;
        C.twall = mess.Twall_ref;
        C.sqrtTwall = std::sqrt(mess.Twall_ref);
        C.vrms = mess.v_rms;
        C.neff = mess.Neff;
        C.dtref = mess.dt_ref;
        C.omega = mess.omega;
        C.eta = mess.eta;
        C.vhsExpF = (float)(1.0 - 2.0 * mess.eta);
        C.expLB = 1.0 / (2.5 - mess.omega);
        C.invAlpha = 1.0 / mess.alpha;
        C.prelaxF = (float)mess.P_relax;
        C.invPrelaxF = mess.P_relax > 0.0 ? (float)(1.0 / mess.P_relax) : 0.0f;
        C.alpha = mess.alpha;
        C.prelax = mess.P_relax;
        C.dr = mess.dr;
        C.nref = mess.n_ref;
        {
            const double conDen = std::tgamma(5.0 / 2.0 - mess.omega);
            const double dref2 = mess.d_ref * mess.d_ref;
            C.cdPrefactor = M_PI * dref2 * std::pow(2 * mess.kB * mess.T_ref / mess.p_mass_r, mess.eta) / conDen;
        }
        C.seedLo = (uint32_t)(params.seed & 0xffffffffu);
        C.seedHi = (uint32_t)(params.seed >> 32);
        C.maxCross = params.max_crossings;
        C.nss = params.nss;
        C.nscheme = params.nscheme;
        C.nevery = params.nevery;
        C.nrepeat = params.nrepeat;
        C.wallStats = params.wall_stats;

        // --- device mesh
        int* dTriOffset; double* dTriD; int2* dTriFT; unsigned char* dRole; int2* dFaceCells;
        int* dFaceWall; double* dWallRot; float* dWallRotF; double* dCenter; double* dVol;
        int* dC2c; signed char* dRev;
        int *dFaceOff; int4* dFaceRec; float4 *dPlaneF, *dDiagF; float2* dRecAux; double* dPlaneD;
        unsigned char* dConvex;
        if (!upload(dFaceOff, faceOff) || !upload(dFaceRec, faceRec) || !upload(dPlaneF, planeF) ||
            !upload(dDiagF, diagF) || !upload(dPlaneD, planeD) || !upload(dConvex, convex) ||
            !upload(dRecAux, recAux))
            return false;
        M.faceOff = dFaceOff; M.faceRec = dFaceRec; M.planeF = dPlaneF; M.diagF = dDiagF; M.planeD = dPlaneD;
        M.convex = dConvex; M.recAux = dRecAux;
        M.faceStride = faceStride;
        M.allConvex = nconvex == ncell ? 1 : 0;
        if (!upload(dTriOffset, triOffset) || !upload(dTriD, triD) || !upload(dTriFT, triFT) ||
            !upload(dRole, roleU8) || !upload(dFaceCells, faceCells) ||
            !upload(dFaceWall, faceWallHost) || !upload(dWallRot, wallRot) || !upload(dWallRotF, wallRotF) ||
            !upload(dCenter, cellCenterHost) || !upload(dVol, vol) || !upload(dC2c, c2c) || !upload(dRev, rev))
            return false;
        M.ncell = ncell; M.nface = nface; M.ntri = ntri; M.nwall = nwall;
        M.triOffset = dTriOffset; M.triD = dTriD; M.triFT = dTriFT;
        M.faceRole = dRole; M.faceCells = dFaceCells; M.faceWall = dFaceWall;
        M.wallRot = dWallRot; M.wallRotF = dWallRotF; M.cellCenter = dCenter; M.cellVolume = dVol;
        M.cell2cell = dC2c; M.revSlot = dRev;
        {
            std::vector<double> placeV;
            buildPlacement(placeV);
            int* dPlaceOff; double* dPlaceV; double* dPlaceVol;
            if (!upload(dPlaceOff, placeOffHost) || !upload(dPlaceV, placeV) || !upload(dPlaceVol, placeVolHost) ||
                !alloc(placeFirst, placeVolHost.size()))
                return false;
            M.placeOff = dPlaceOff; M.placeV = dPlaceV; M.placeVol = dPlaceVol;
        }

        // --- per-cell state (Collision_constant_initial, src/MeshparticalInitial.cpp:798-810)
        std::vector<double> crInit((size_t)ncell, 3.0);
        if (!upload(crmax, crInit)) return false;
        if (!alloc(remColl, (size_t)ncell) || !alloc(remInj, (size_t)ncell) || !alloc(acc, (size_t)ncell * 54) ||
            !alloc(record, (size_t)ncell * 18) || !alloc(local, (size_t)ncell * 18) ||
            !alloc(finalRecord, (size_t)ncell * 18) || !alloc(sparseState, (size_t)ncell) ||
            !alloc(sparseAccum, (size_t)ncell) || !alloc(windowSamples, (size_t)ncell) ||
            !alloc(windowValid, (size_t)ncell) || !alloc(wallTally, (size_t)std::max(nwall, 1) * 6) ||
            !alloc(countSlot, (size_t)ncell * kSlots) || !alloc(scanPartial, kScanBlocks) ||
            !alloc(start[0], (size_t)ncell + 1) || !alloc(start[1], (size_t)ncell + 1) || !alloc(ctl, 1) ||
            !alloc(counters, C_COUNT) || !alloc(cellList, (size_t)ncell * 2) || !alloc(cellWork, 8) ||
            !alloc(cellPairs, (size_t)ncell) || !alloc(cellCons, (size_t)ncell) ||
            !alloc(cellItem, (size_t)ncell) || !alloc(cellItemC, (size_t)ncell) ||
            !alloc(errorWord, 1) || !alloc(uploadFlag, 1))
            return false;
        if (params.keep_step_moments && !alloc(stepMom, (size_t)ncell * 18)) return false;
        cudaError_t pe = (precision == DSMC_PRECISION_MIXED) ? prepare_kernels<float>() : prepare_kernels<double>();
        if (!cuda(pe, "kernel attributes")) return false;
        for (auto& e : ev)
            if (!cuda(cudaEventCreate(&e), "cudaEventCreate")) return false;
        if (params.capacity > 0 && !ensureCapacity(params.capacity)) return false;
        return cuda(cudaStreamSynchronize(stream), "create sync");
    }

    bool buildPatches()
    {
        struct Patch {
            int cell, edge, tag;
            double geom[9], rot[9], gas[8], addBase;
        };
        std::vector<Patch> patches;
        const double gamma = mess.gamma;
        for (int f = 0; f < nface; ++f) {
            bool inject = false;
            const int role = roleOfTag(edges[(size_t)f].faceTag, &inject);
            if (role != DSMC_ROLE_INLET || !inject) continue;
            const DsmcEdgeRec& edge = edges[(size_t)f];
            const int g1 = edge.faceMap[4], g2 = edge.faceMap[5];
            int cellLocal = -1;
            if (g1 >= 0 && g1 < ncell) cellLocal = g1;
            if (cellLocal < 0 && g2 >= 0 && g2 < ncell) cellLocal = g2;
            if (cellLocal < 0) continue;
            const int faceType = edge.faceType;
            if (faceType != 3 && faceType != 4) continue;
            const int nodeCount = faceType == 4 ? 4 : 3;
            double pts[4][3];
            bool ok = true;
            for (int k = 0; k < nodeCount && ok; ++k) ok = loadPoint(edge.faceMap[k], pts[k]);
            if (!ok) continue;
            int tri[2][3] = {{0, 1, 2}, {-1, -1, -1}};
            int nTris = 1;
            double qn[2][3] = {};
            if (faceType == 4) {
                int t0[3], t1[3];
                decode_split(split[(size_t)f], t0, t1);
                if (t0[0] < 0 || t1[0] < 0) decode_split(kSplit02, t0, t1);
                for (int k = 0; k < 3; ++k) { tri[0][k] = t0[k]; tri[1][k] = t1[k]; }
                nTris = 2;
                // wallMap normals (processFacesQuadNormals over inletVisMove)
                for (int s = 0; s < 2; ++s) {
                    const int* tt = tri[s];
                    const double* X = pts[tt[0]];
                    const double* Y = pts[tt[1]];
                    const double* Z = pts[tt[2]];
                    const double e1[3] = {Y[0] - X[0], Y[1] - X[1], Y[2] - X[2]};
                    const double e2[3] = {Z[0] - X[0], Z[1] - X[1], Z[2] - X[2]};
                    cross3(e1, e2, qn[s]);
                    normalize3(qn[s]);
                    if (dot3(edge.edgeNormal, qn[s]) < 0.0) {
                        qn[s][0] *= -1.0; qn[s][1] *= -1.0; qn[s][2] *= -1.0;
                    }
                }
            }
            for (int tagTri = 1; tagTri <= nTris; ++tagTri) {
                const int slot = faceType == 4 ? tagTri - 1 : 0;
                double norm[3];
                if (faceType == 4) {
                    for (int d = 0; d < 3; ++d) norm[d] = qn[slot][d];
                } else {
                    for (int d = 0; d < 3; ++d) norm[d] = edge.edgeNormal[d];
                    const double len = std::sqrt(norm[0] * norm[0] + norm[1] * norm[1] + norm[2] * norm[2]);
                    if (len > 0.0 && std::isfinite(len)) { norm[0] /= len; norm[1] /= len; norm[2] /= len; }
                }
                const double* P0 = pts[tri[slot][0]];
                const double* P1 = pts[tri[slot][1]];
                const double* P2 = pts[tri[slot][2]];
                Patch pt{};
                pt.cell = cellLocal;
                pt.edge = f;
                pt.tag = faceType == 3 ? -1 : tagTri;
                for (int d = 0; d < 3; ++d) {
                    pt.geom[d] = P0[d];
                    pt.geom[3 + d] = P1[d] - P0[d];
                    pt.geom[6 + d] = P2[d] - P0[d];
                }
                // triangleArea, src/ProcessDSMC.cpp:601-614
                const double ax = P1[0] - P0[0], ay = P1[1] - P0[1], az = P1[2] - P0[2];
                const double bx = P2[0] - P0[0], by = P2[1] - P0[1], bz = P2[2] - P0[2];
                const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
                const double area = 0.5 * std::sqrt(cx * cx + cy * cy + cz * cz);
                const double nmag = std::sqrt(norm[0] * norm[0] + norm[1] * norm[1] + norm[2] * norm[2]);
                if (!(area > 0.0) || !std::isfinite(area) || !(nmag > 0.0) || !std::isfinite(nmag)) continue;
                double neg[3] = {-norm[0], -norm[1], -norm[2]};
                double R[9];
                rotation(neg, R);
                for (int k = 0; k < 9; ++k) pt.rot[k] = R[k];
                // computeBoundaryGasState, src/ProcessDSMC.cpp:2318-2367 (FreestreamInlet)
                const double base = 1.0 * mess.Ma * std::sqrt(gamma / 2.0) * mess.v_in / mess.v_rms;
                const double uxN = base * params.inflow_dir[0];
                const double uyN = base * params.inflow_dir[1];
                const double uzN = 0.0;
                const double tN = mess.T_in / mess.T_ref;
                const double rhoP = 1.0 * mess.n_ref;
                const double uxP = uxN * mess.v_rms, uyP = uyN * mess.v_rms, uzP = uzN * mess.v_rms;
                const double tP = tN * mess.T_ref;
                const double beta = 1.0 / std::sqrt(2 * mess.kB / mess.p_mass * tP);
                const double sx = uxP * beta, sy = uyP * beta, sz = uzP * beta;
                // rotation[i][j] = R[3i+j]
                const double stp1 = R[0] * sx + R[3] * sy + R[6] * sz;
                const double stp2 = R[1] * sx + R[4] * sy + R[7] * sz;
                const double snp = R[2] * sx + R[5] * sy + R[8] * sz;
                const double fs1 = snp + std::sqrt(snp * snp + 2.0);
                const double fs2 = 0.5 * (1.0 + snp * (2.0 * snp - fs1));
                double QA = 3.0;
                if (std::fabs(snp) > 3.0) QA = std::fabs(snp) + 1.0;
                pt.gas[0] = snp; pt.gas[1] = fs1; pt.gas[2] = fs2; pt.gas[3] = stp1; pt.gas[4] = stp2;
                pt.gas[5] = tN; pt.gas[6] = std::sqrt(tN); pt.gas[7] = QA;
                // computeBoundaryInsertCount, src/ProcessDSMC.cpp:2380-2403
                double cosTheta = 0.0;
                const double Umag = std::sqrt(uxP * uxP + uyP * uyP + uzP * uzP);
                if (Umag > 0.0 && nmag > 0.0)
                    cosTheta = -((uxP * norm[0] + uyP * norm[1] + uzP * norm[2]) / (Umag * nmag));
                const double s = beta * Umag;
                const double scos = s * cosTheta;
                double addNum = mess.dtime * area * rhoP / 2.0 / std::sqrt(M_PI) * std::sqrt(tP / mess.T_ref) *
                                (std::exp(-(scos * scos)) + std::sqrt(M_PI) * scos * (1.0 + std::erf(scos)));
                pt.addBase = addNum / mess.Neff;
                if (!std::isfinite(pt.addBase) || pt.addBase < 0.0 || pt.addBase > 1.0e8)
                    return fail("inflow patch count out of range");
                patches.push_back(pt);
            }
        }
        // group patches by cell, keeping their order within a cell
        std::stable_sort(patches.begin(), patches.end(), [](const Patch& a, const Patch& b) { return a.cell < b.cell; });
        const int np = (int)patches.size();
        std::vector<int> groupStart;
        std::vector<int> pc(np), pe(np), ptg(np);
        std::vector<double> geom((size_t)np * 9), rot((size_t)np * 9), gas((size_t)np * 8), addBase(np);
        for (int i = 0; i < np; ++i) {
            if (i == 0 || patches[(size_t)i].cell != patches[(size_t)i - 1].cell) groupStart.push_back(i);
            pc[(size_t)i] = patches[(size_t)i].cell;
            pe[(size_t)i] = patches[(size_t)i].edge;
            ptg[(size_t)i] = patches[(size_t)i].tag;
            std::memcpy(&geom[(size_t)i * 9], patches[(size_t)i].geom, 9 * sizeof(double));
            std::memcpy(&rot[(size_t)i * 9], patches[(size_t)i].rot, 9 * sizeof(double));
            std::memcpy(&gas[(size_t)i * 8], patches[(size_t)i].gas, 8 * sizeof(double));
            addBase[(size_t)i] = patches[(size_t)i].addBase;
        }
        const int ngroup = (int)groupStart.size();
        groupStart.push_back(np);
        int *dG, *dC, *dE, *dT, *dCount, *dStart;
        double *dGeom, *dRot, *dGas, *dAdd;
        if (!upload(dG, groupStart) || !upload(dC, pc) || !upload(dE, pe) || !upload(dT, ptg) || !upload(dGeom, geom) ||
            !upload(dRot, rot) || !upload(dGas, gas) || !upload(dAdd, addBase) || !alloc(dCount, (size_t)np) ||
            !alloc(dStart, (size_t)np))
            return false;
        P.npatch = np; P.ngroup = ngroup; P.groupStart = dG; P.cell = dC; P.edge = dE; P.triTag = dT;
        P.geom = dGeom; P.rot = dRot; P.gas = dGas; P.addBase = dAdd; P.count = dCount; P.start = dStart;
        return true;
    }

    bool ensureCapacity(int64_t need)
    {
        if (need <= capacity) return true;
        if (need > (int64_t)0x7fffffff - 1) return fail("capacity above 2^31 particles");
        // keep existing particles
        std::vector<std::vector<char>> keep;
        const size_t rs = realSize();
        int n = haveParticles ? hostNLive : 0;
        if (n > 0) {
            keep.resize(8);
            for (int k = 0; k < 8; ++k) {
                const size_t es = (k == 7) ? sizeof(int) : rs;
                keep[(size_t)k].resize((size_t)n * es);
                if (!cuda(cudaMemcpyAsync(keep[(size_t)k].data(), buf[cur][k], (size_t)n * es, cudaMemcpyDeviceToHost, stream), "keep"))
                    return false;
            }
            if (!cuda(cudaStreamSynchronize(stream), "keep sync")) return false;
        }
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 8; ++k) { freePtr(buf[b][k]); buf[b][k] = nullptr; }
        freePtr(rank); freePtr(idx);
        rank = nullptr; idx = nullptr;
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        ++generation;
        const int64_t cap = need;
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 8; ++k) {
                char* p = nullptr;
                const size_t es = (k == 7) ? sizeof(int) : rs;
                if (!alloc(p, (size_t)cap * es, false)) return false;
                buf[b][k] = p;
            }
        if (!alloc(rank, (size_t)cap, false) || !alloc(idx, (size_t)cap, true)) return false;
        capacity = cap;
        for (int k = 0; k < 8 && n > 0; ++k) {
            const size_t es = (k == 7) ? sizeof(int) : rs;
            if (!cuda(cudaMemcpyAsync(buf[cur][k], keep[(size_t)k].data(), (size_t)n * es, cudaMemcpyHostToDevice, stream), "restore"))
                return false;
        }
        StepCtl h{};
        h.nLive = n;
        h.capacity = (int)capacity;
        if (!cuda(cudaMemcpyAsync(ctl, &h, sizeof h, cudaMemcpyHostToDevice, stream), "ctl")) return false;
        return cuda(cudaStreamSynchronize(stream), "capacity sync");
    }

    template <typename Real>
    StepArgs<Real> args() const
    {
        StepArgs<Real> a{};
        a.M = M; a.C = C; a.P = P;
        const int o = cur ^ 1;
        for (int d = 0; d < 3; ++d) {
            a.A.x[d] = (Real*)buf[cur][d];
            a.A.v[d] = (Real*)buf[cur][3 + d];
            a.B.x[d] = (Real*)buf[o][d];
            a.B.v[d] = (Real*)buf[o][3 + d];
        }
        a.A.ir = (Real*)buf[cur][6]; a.A.cell = (int*)buf[cur][7];
        a.B.ir = (Real*)buf[o][6]; a.B.cell = (int*)buf[o][7];
        a.startA = start[cur]; a.startB = start[o];
        a.rank = rank; a.idx = idx; a.countSlot = countSlot; a.scanPartial = scanPartial;
        a.crmax = crmax; a.remColl = remColl; a.remInj = remInj; a.acc = acc; a.record = record;
        a.local = local; a.finalRecord = finalRecord; a.stepMom = stepMom;
        a.sparseState = sparseState; a.sparseAccum = sparseAccum; a.windowSamples = windowSamples;
        a.windowValid = windowValid; a.wallTally = wallTally; a.ctl = ctl; a.counters = counters;
        a.cellList = cellList; a.cellWork = cellWork; a.errorWord = errorWord;
        a.cellPairs = cellPairs; a.cellCons = cellCons;
        a.cellItem = cellItem; a.cellItemC = cellItemC;
        return a;
    }

    bool setIstep(int istep)
    {
        return cuda(cudaMemcpyAsync(&ctl->istep, &istep, sizeof(int), cudaMemcpyHostToDevice, stream), "istep");
    }

    // Enqueue the selected stages. Returns with `cur` flipped if a sort ran.
    template <typename Real>
    void enqueue(uint32_t stages, bool events)
    {
        const StepArgs<Real> a = args<Real>();
        if (events) cudaEventRecord(ev[0], stream);
        if (stages & DSMC_STAGE_INJECT) launch_inject<Real>(a, shape, stream);
        if (events) cudaEventRecord(ev[1], stream);
        if (stages & DSMC_STAGE_MOVE) launch_move<Real>(a, shape, stream);
        if (events) cudaEventRecord(ev[2], stream);
        const bool sort = (stages & DSMC_STAGE_SORT) != 0;
        const bool coll = (stages & DSMC_STAGE_COLLIDE) != 0;
        const bool samp = (stages & DSMC_STAGE_SAMPLE) != 0;
        if (sort) {
            // rank, scan, scatter, far-slot order, gather into B
            launch_sort<Real>(a, shape, stream);
            cudaMemcpyAsync(&ctl->nLive, &ctl->nNext, sizeof(int), cudaMemcpyDeviceToDevice, stream);
            cudaMemsetAsync(&ctl->nInj, 0, sizeof(int), stream);
        }
        if (events) cudaEventRecord(ev[3], stream);
        // collisions and sampling act in place on the (now) current buffer
        StepArgs<Real> b = a;
        if (sort) {
            b.A = a.B; b.B = a.A; b.startA = a.startB; b.startB = const_cast<int*>(a.startA);
        }
        if (coll) launch_collide<Real>(b, shape, stream);
        if (events) cudaEventRecord(ev[4], stream);
        if (samp) launch_sample<Real>(b, false, shape, stream);
        if (events) cudaEventRecord(ev[5], stream);
    }

    template <typename Real>
    bool stepT(int istep, uint32_t stages)
    {
        if (!haveParticles) return fail("no particles uploaded");
        if (stages & ~DSMC_STAGE_ALL) return fail("unknown stage flags");
        if (!setIstep(istep)) return false;
        curIstep = istep;
        devIstepValid = true;
        const bool full = stages == DSMC_STAGE_ALL;
        if (full && !timing && std::getenv("DSMC_NO_GRAPH") == nullptr) {
            if (!graph[cur]) {
                cudaGraph_t g = nullptr;
                if (!cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "capture")) return false;
                enqueue<Real>(stages, false);
                if (!cuda(cudaStreamEndCapture(stream, &g), "end capture")) return false;
                const cudaError_t ie = cudaGraphInstantiate(&graph[cur], g, 0);
                cudaGraphDestroy(g);
                if (!cuda(ie, "graph instantiate")) return false;
            }
            if (!cuda(cudaGraphLaunch(graph[cur], stream), "graph launch")) return false;
        } else {
            enqueue<Real>(stages, timing);
            if (!cuda(cudaGetLastError(), "kernel launch")) return false;
            if (timing) {
                if (!cuda(cudaEventSynchronize(ev[5]), "timing sync")) return false;
                for (int k = 0; k < 5; ++k) {
                    float ms = 0.0f;
                    cudaEventElapsedTime(&ms, ev[k], ev[k + 1]);
                    stageMs[k] += ms;
                }
                ++timedSteps;
            }
        }
        if (stages & DSMC_STAGE_INJECT) pendingInject = true;
        if (stages & DSMC_STAGE_SORT) {
            cur ^= 1;
            pendingInject = false;
        }
        if (stages & DSMC_STAGE_SAMPLE) {
            localLazy = true;
            lastIstep = istep;
        }
        if (stages & DSMC_STAGE_MOVE) ++steps;
        return true;
    }

    bool step(int istep, uint32_t stages)
    {
        return precision == DSMC_PRECISION_MIXED ? stepT<float>(istep, stages) : stepT<double>(istep, stages);
    }

    void dropGraphs()
    {
        for (auto& g : graph)
            if (g) { cudaGraphExecDestroy(g); g = nullptr; }
        ++generation;
    }

    bool setShape(const DsmcLaunchShape& s)
    {
        if (s.move_threads != 128 && s.move_threads != 256)
            return fail("launch shape: move_threads must be 128 or 256");
        if (s.move_blocks_per_sm < 1 || s.move_blocks_per_sm > 32 || s.sort_blocks_per_sm < 1 ||
            s.sort_blocks_per_sm > 32 || s.collide_blocks_per_sm < 1 || s.collide_blocks_per_sm > 32)
            return fail("launch shape: blocks per SM outside [1, 32]");
        if (s.stay_per_thread != 1 && s.stay_per_thread != 2 && s.stay_per_thread != 4)
            return fail("launch shape: stay_per_thread must be 1, 2 or 4");
        // work already queued keeps the shape it was launched with
        shape.moveThreads = s.move_threads;
        shape.moveBlocksPerSm = s.move_blocks_per_sm;
        shape.sortBlocksPerSm = s.sort_blocks_per_sm;
        shape.collideBlocksPerSm = s.collide_blocks_per_sm;
        shape.stayPerThread = s.stay_per_thread;
        dropGraphs();
        return true;
    }

    DsmcLaunchShape getShape() const
    {
        DsmcLaunchShape s;
        s.move_threads = shape.moveThreads;
        s.move_blocks_per_sm = shape.moveBlocksPerSm;
        s.sort_blocks_per_sm = shape.sortBlocksPerSm;
        s.collide_blocks_per_sm = shape.collideBlocksPerSm;
        s.stay_per_thread = shape.stayPerThread;
        return s;
    }

    // The autotuner: runs full steps of this case from step `istep` on,
    // timing each stage with events, and keeps per stage the fastest of a
    // few launch shapes (move: block size x blocks per SM, particles per
    // thread of the stay pass; rank / scatter / gather: blocks per SM).
    // Since no kernel's
    // result depends on its launch shape, the steps it runs are ordinary
    // steps of the case; on return `istep` is the next step to run.
    bool autotune(int& istep, int trialSteps)
    {
        if (trialSteps < 1) return fail("autotune: trial_steps < 1");
        const bool wasTiming = timing;
        timing = true;
        auto trial = [&](const DsmcLaunchShape& cand, int stage, double& ms) -> bool {
            if (!setShape(cand)) return false;
            for (double& v : stageMs) v = 0.0;
            timedSteps = 0;
            for (int k = 0; k < trialSteps; ++k)
                if (!step(istep++, DSMC_STAGE_ALL)) return false;
            ms = stageMs[stage] / (double)trialSteps;
            return true;
        };
        DsmcLaunchShape best = getShape();
        bool ok = step(istep++, DSMC_STAGE_ALL);   // one untimed-order step to warm the caches
        double bestMs = 0.0;
        if (ok) ok = trial(best, 1, bestMs);
        const int threads[2] = {128, 256};
        const int blocks[4] = {2, 4, 8, 16};
        for (int t = 0; ok && t < 2; ++t)
            for (int b = 0; ok && b < 4; ++b) {
                DsmcLaunchShape c = best;
                c.move_threads = threads[t];
                c.move_blocks_per_sm = blocks[b] * 256 / threads[t] > 0 ? blocks[b] * 256 / threads[t] : 1;
                if (c.move_threads == best.move_threads && c.move_blocks_per_sm == best.move_blocks_per_sm) continue;
                double ms = 0.0;
                ok = trial(c, 1, ms);
                if (ok && ms < bestMs) { bestMs = ms; best = c; }
            }
        const int perThread[3] = {1, 2, 4};
        for (int k = 0; ok && k < 3; ++k) {
            DsmcLaunchShape c = best;
            c.stay_per_thread = perThread[k];
            if (c.stay_per_thread == best.stay_per_thread) continue;
            double ms = 0.0;
            ok = trial(c, 1, ms);
            if (ok && ms < bestMs) { bestMs = ms; best = c; }
        }
        if (ok) ok = trial(best, 2, bestMs);
        for (int b = 0; ok && b < 4; ++b) {
            DsmcLaunchShape c = best;
            c.sort_blocks_per_sm = blocks[b];
            if (c.sort_blocks_per_sm == best.sort_blocks_per_sm) continue;
            double ms = 0.0;
            ok = trial(c, 2, ms);
            if (ok && ms < bestMs) { bestMs = ms; best = c; }
        }
        // collide keeps its grid cap (the resident-block maximum by
        // default): fewer blocks per SM were slower in every timed run, and
        // single-step trials of them picked them by noise
        timing = wasTiming;
        for (double& v : stageMs) v = 0.0;
        timedSteps = 0;
        if (!ok) return false;
        return setShape(best);
    }

    // ---- batched steps (DsmcBatch): one full step on the handle's stream,
    // the step counter advanced on the device, recorded into the batch graph
    template <typename Real>
    void enqueueBatchT()
    {
        launch_bump_istep(ctl, stream);
        enqueue<Real>(DSMC_STAGE_ALL, false);
    }
    void enqueueBatch()
    {
        if (precision == DSMC_PRECISION_MIXED) enqueueBatchT<float>();
        else enqueueBatchT<double>();
    }
    void afterBatchStep()
    {
        ++curIstep;
        cur ^= 1;
        pendingInject = false;
        localLazy = true;
        lastIstep = curIstep;
        ++steps;
    }

    bool macroPre()
    {
        if (!haveParticles) return fail("no particles uploaded");
        if (precision == DSMC_PRECISION_MIXED) launch_sample<float>(args<float>(), true, shape, stream);
        else launch_sample<double>(args<double>(), true, shape, stream);
        localLazy = false;
        return cuda(cudaGetLastError(), "statistic_macroPre");
    }

    bool nLiveHost(int& n)
    {
        if (!cuda(cudaMemcpyAsync(&n, &ctl->nLive, sizeof(int), cudaMemcpyDeviceToHost, stream), "nLive")) return false;
        if (!cuda(cudaStreamSynchronize(stream), "sync")) return false;
        hostNLive = n;
        return true;
    }

    bool checkDeviceErrors()
    {
        int e = 0;
        if (!cuda(cudaMemcpyAsync(&e, errorWord, sizeof(int), cudaMemcpyDeviceToHost, stream), "error word")) return false;
        if (!cuda(cudaStreamSynchronize(stream), "sync")) return false;
        if (e & kErrRejectLoop) return fail("inflow sampling rejection loop exceeded its bound");
        if (e & kErrSortIndex) return fail("device self-check: inconsistent sort index (error word 8)");
        if (e & kErrStageCell) return fail("device self-check: a cell larger than the shared stage (error word 2)");

        return true;
    }

    // Whether host memory is page-locked (or registered), so the DMA engine
    // can read it in place.
    static bool hostPinned(const void* p)
    {
        cudaPointerAttributes a{};
        if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
            (void)cudaGetLastError();
            return false;
        }
        return a.type == cudaMemoryTypeHost;
    }

    // Host -> device on the handle's stream: pinned memory in one copy;
    // pageable memory through the two pinned chunks, the host copy of the
    // next chunk overlapping the transfer of the last. The source may be
    // reused once the stream has been synchronised.
    bool h2d(void* dst, const void* src, size_t bytes)
    {
        if (bytes == 0) return true;
        if (hostPinned(src)) return cuda(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream), "upload");
        for (int b = 0; b < 2; ++b) {
            if (!hostStage[b] && !cuda(cudaHostAlloc(&hostStage[b], kHostStage, cudaHostAllocDefault), "pinned staging"))
                return false;
            if (!stageEv[b] && !cuda(cudaEventCreateWithFlags(&stageEv[b], cudaEventDisableTiming), "staging event"))
                return false;
        }
        const char* s = static_cast<const char*>(src);
        char* d = static_cast<char*>(dst);
        const int nthreads = hostpack::threads_for((int64_t)(kHostStage / 8));
        size_t j = 0;
        for (size_t off = 0; off < bytes; off += kHostStage, ++j) {
            const int b = (int)(j & 1);
            const size_t len = std::min(kHostStage, bytes - off);
            if (!cuda(cudaEventSynchronize(stageEv[b]), "staging wait")) return false;
            hostpack::parallel_copy(hostStage[b], s + off, len, nthreads);
            if (!cuda(cudaMemcpyAsync(d + off, hostStage[b], len, cudaMemcpyHostToDevice, stream), "upload") ||
                !cuda(cudaEventRecord(stageEv[b], stream), "staging event"))
                return false;
        }
        return true;
    }

    // Upload of particles already in cell-major order (the order of the
    // reference's per-cell buckets, and of dsmc_download_particles): the cell
    // ids go up first and a kernel checks them and lays out start[]; the
    // columns then go up unchanged (FP64) or through the other particle
    // buffer, chunk by chunk, into FP32 offsets from the cell centres (mixed).
    // Returns 1 when done, 0 when the cells are not in that order (nothing
    // is kept; the caller orders them on the host), -1 on an error.
    int uploadCellMajor(int64_t n, const double* const src[7], const int32_t* cell)
    {
        int* dCell = static_cast<int*>(buf[cur][7]);
        if (!h2d(dCell, cell, (size_t)n * sizeof(int))) return -1;
        if (!cuda(cudaMemsetAsync(uploadFlag, 0, sizeof(int), stream), "upload flag")) return -1;
        launch_upload_check(dCell, (int)n, ncell, uploadFlag, start[cur], stream);
        int flags = 0;
        if (!cuda(cudaGetLastError(), "upload check") ||
            !cuda(cudaMemcpyAsync(&flags, uploadFlag, sizeof(int), cudaMemcpyDeviceToHost, stream), "upload flag") ||
            !cuda(cudaStreamSynchronize(stream), "upload check sync"))
            return -1;
        if (flags & 1) {
            fail("particle cell id out of range");
            return -1;
        }
        if (flags & 2) return 0;
        if (precision != DSMC_PRECISION_MIXED) {
            for (int k = 0; k < 7; ++k)
                if (!h2d(buf[cur][k], src[k], (size_t)n * sizeof(double))) return -1;
            return 1;
        }
        // device chunks of the FP64 columns: the x and y arrays of the other
        // buffer (capacity FP32 slots each, capacity / 2 FP64 values)
        const int64_t m = std::max<int64_t>(1, capacity / 2);
        double* dstage[2] = {static_cast<double*>(buf[cur ^ 1][0]), static_cast<double*>(buf[cur ^ 1][1])};
        int64_t j = 0;
        for (int k = 0; k < 7; ++k) {
            float* out = static_cast<float*>(buf[cur][k]);
            for (int64_t off = 0; off < n; off += m, ++j) {
                const int64_t len = std::min(m, n - off);
                double* ds = dstage[j & 1];
                if (!h2d(ds, src[k] + off, (size_t)len * sizeof(double))) return -1;
                launch_upload_convert(ds, dCell + off, M.cellCenter, k, out + off, (int)len, stream);
            }
        }
        return cuda(cudaGetLastError(), "upload convert") ? 1 : -1;
    }

    bool uploadParticles(int64_t n, const double* px, const double* py, const double* pz, const double* vx,
                         const double* vy, const double* vz, const double* ir, const int32_t* cell)
    {
        if (n < 0) return fail("negative particle count");
        if (n > (int64_t)0x7fffffff - 1) return fail("capacity above 2^31 particles");
        if (n > 0 && (!px || !py || !pz || !vx || !vy || !vz || !ir || !cell)) return fail("null particle array");
        const double* src[7] = {px, py, pz, vx, vy, vz, ir};
        if (n > 0) {
            const int64_t need = params.capacity > 0 ? params.capacity : std::max<int64_t>(n + n / 2 + (1 << 16), 1 << 20);
            if (n > need) return fail("more particles than the configured capacity");
            haveParticles = false;
            if (!ensureCapacity(need)) return false;
            const int r = uploadCellMajor(n, src, cell);
            if (r < 0) return false;
            if (r == 1) return finishUpload(n);
        }
        const int nthreads = hostpack::threads_for(n);
        if (!hostpack::cells_in_range(n, cell, ncell, nthreads)) return fail("particle cell id out of range");
        // order: cell-major, input order within a cell
        std::vector<int> st;
        std::vector<int64_t> order;
        hostpack::order_by_cell(n, cell, ncell, nthreads, st, order);
        int64_t need = params.capacity > 0 ? params.capacity : std::max<int64_t>(n + n / 2 + (1 << 16), 1 << 20);
        if (n > need) return fail("more particles than the configured capacity");
        haveParticles = false;
        if (!ensureCapacity(need)) return false;
        const bool mixed = precision == DSMC_PRECISION_MIXED;
        std::vector<char> hb((size_t)n * 8);
        for (int k = 0; k < 7; ++k) {
            if (mixed)
                hostpack::gather_convert<float>(n, order.data(), src[k], cell, k < 3 ? cellCenterHost.data() : nullptr, k,
                                                reinterpret_cast<float*>(hb.data()), nthreads);
            else
                hostpack::gather_convert<double>(n, order.data(), src[k], cell, nullptr, k,
                                                 reinterpret_cast<double*>(hb.data()), nthreads);
            if (n > 0 && (!cuda(cudaMemcpyAsync(buf[cur][k], hb.data(), (size_t)n * realSize(), cudaMemcpyHostToDevice, stream), "upload particles") ||
                          !cuda(cudaStreamSynchronize(stream), "sync")))
                return false;
        }
        std::vector<int> hc((size_t)n);
        hostpack::gather_cells(n, order.data(), cell, hc.data(), nthreads);
        if (n > 0 && !cuda(cudaMemcpyAsync(buf[cur][7], hc.data(), (size_t)n * sizeof(int), cudaMemcpyHostToDevice, stream), "upload cells"))
            return false;
        if (!cuda(cudaMemcpyAsync(start[cur], st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice, stream), "upload start"))
            return false;
        return finishUpload(n);
    }

    bool finishUpload(int64_t n)
    {
        StepCtl h{};
        h.nLive = (int)n;
        h.capacity = (int)capacity;
        if (!cuda(cudaMemcpyAsync(ctl, &h, sizeof h, cudaMemcpyHostToDevice, stream), "ctl")) return false;
        if (!cuda(cudaMemsetAsync(countSlot, 0, (size_t)ncell * kSlots * sizeof(int), stream), "countSlot")) return false;
        if (!cuda(cudaStreamSynchronize(stream), "upload sync")) return false;
        hostNLive = (int)n;
        haveParticles = true;
        devIstepValid = false;
        pendingInject = false;
        return true;
    }

    // Device-side initial fill. Counts follow setParticleMessage
    // (src/meshImport.cpp:1399-1421): cell c expects Ns = V_c * Nps / V_total
    // particles (Nps = ppcMean * ncell) and gets floor(Ns) + 1 with
    // probability frac(Ns), else floor(Ns); the draw for cell c is Philox
    // counter (c, 0, kPurposeFillCount, 0) under the key `seed`. Placement and
    // velocities: fill_kernel.
    // Sub-tetrahedron counts of one cell (Np_tri_inititial,
    // src/MeshparticalInitial.cpp:481-514): Iround(Np V_t / V_cell) each,
    // then adjust_particles (src/MeshparticalInitial.cpp:752-786) moves the
    // sum to Np by +-1 on |delta| distinct tetrahedra chosen by a partial
    // Fisher-Yates shuffle (all of them when |delta| reaches their number)
    // and clamps at zero. Draws: Philox (c, t, kPurposeFillCount, 1) for the
    // rounding of tetrahedron t, (c, i, kPurposeFillCount, 2) for shuffle
    // step i. Returns the cell's particle count.
    static int subTetCounts(int c, int np, const double* vol, int nt, uint32_t k0, uint32_t k1, int* first)
    {
        if (np <= 0 || nt <= 0) {
            for (int t = 0; t < nt; ++t) first[t] = 0;
            return 0;
        }
        double sumVol = 0.0;
        for (int t = 0; t < nt; ++t) sumVol += vol[t];
        std::vector<double> region((size_t)nt);
        int sumN = 0;
        for (int t = 0; t < nt; ++t) {
            const double x = static_cast<double>(np) * vol[t] / sumVol;
            const double fl = std::floor(x);
            const U4 b = philox4x32_10(U4{(uint32_t)c, (uint32_t)t, kPurposeFillCount, 1u}, k0, k1);
            region[(size_t)t] = (unit64(b.x, b.y) < x - fl) ? fl + 1.0 : fl;
            sumN += static_cast<int>(region[(size_t)t]);
        }
        const int delta = np - sumN;
        const int absDelta = std::abs(delta);
        const double step = delta > 0 ? 1.0 : -1.0;
        if (absDelta >= nt) {
            for (int t = 0; t < nt; ++t) region[(size_t)t] += step;
        } else if (absDelta > 0) {
            std::vector<int> ind((size_t)nt);
            for (int t = 0; t < nt; ++t) ind[(size_t)t] = t;
            for (int i = 0; i < absDelta; ++i) {
                const U4 b = philox4x32_10(U4{(uint32_t)c, (uint32_t)i, kPurposeFillCount, 2u}, k0, k1);
                int r = i + (int)(unit64(b.x, b.y) * (double)(nt - i));
                if (r > nt - 1) r = nt - 1;
                std::swap(ind[(size_t)i], ind[(size_t)r]);
            }
            for (int i = 0; i < absDelta; ++i) region[(size_t)ind[(size_t)i]] += step;
        }
        int n = 0;
        for (int t = 0; t < nt; ++t) {
            first[t] = n;
            n += static_cast<int>(std::max(region[(size_t)t], 0.0));
        }
        return n;
    }

    // The initial fill (Np_tri_inititial / meshfillpar, src/MeshparticalInitial.cpp:
    // 413-418, 481-721) with the per-cell counts of setParticleMessage
    // (src/meshImport.cpp:1399-1421). atRest: the reference's unit Maxwellian
    // at rest; otherwise the case's freestream.
    bool fill(double ppcMean, uint64_t seed, bool atRest)
    {
        if (!(ppcMean > 0.0) || !std::isfinite(ppcMean)) return fail("fill: particles per cell must be positive");
        const uint32_t k0 = (uint32_t)(seed & 0xffffffffu), k1 = (uint32_t)(seed >> 32);
        double vtot = 0.0;
        for (int c = 0; c < ncell; ++c) vtot += cells[(size_t)c].area;
        if (!(vtot > 0.0)) return fail("fill: zero mesh volume");
        const double nps = ppcMean * (double)ncell;
        std::vector<int> st((size_t)ncell + 1, 0);
        std::vector<int> first(placeVolHost.size(), 0);
        int64_t total = 0;
        for (int c = 0; c < ncell; ++c) {
            const double ns = cells[(size_t)c].area * nps / vtot;
            const double fl = std::floor(ns);
            if (!(fl < 1.0e9)) return fail("fill: more than 1e9 particles in a cell");
            const U4 b = philox4x32_10(U4{(uint32_t)c, 0u, kPurposeFillCount, 0u}, k0, k1);
            const int np = (int)fl + ((unit64(b.x, b.y) < ns - fl) ? 1 : 0);
            const int t0 = placeOffHost[(size_t)c], nt = placeOffHost[(size_t)c + 1] - t0;
            total += subTetCounts(c, np, placeVolHost.data() + t0, nt, k0, k1, first.data() + t0);
            if (total > (int64_t)0x7fffffff - 1) return fail("fill: more than 2^31 particles");
            st[(size_t)c + 1] = (int)total;
        }
        const int64_t need = params.capacity > 0 ? params.capacity
                                                 : std::max<int64_t>(total + total / 2 + (1 << 16), 1 << 20);
        if (total > need) return fail("fill: more particles than the configured capacity");
        haveParticles = false;
        if (!ensureCapacity(need)) return false;
        if (!cuda(cudaMemcpyAsync(start[cur], st.data(), st.size() * sizeof(int), cudaMemcpyHostToDevice, stream), "fill start"))
            return false;
        if (!first.empty() &&
            !cuda(cudaMemcpyAsync(placeFirst, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice, stream),
                  "fill tetrahedra"))
            return false;
        FillParams f{};
        if (atRest) {
            f.sig = 1.0;
            f.tN = 1.0;
        } else {
            const double base = 1.0 * mess.Ma * std::sqrt(mess.gamma / 2.0) * mess.v_in / mess.v_rms;
            f.u[0] = base * params.inflow_dir[0];
            f.u[1] = base * params.inflow_dir[1];
            f.u[2] = 0.0;
            f.tN = mess.T_in / mess.T_ref;
            f.sig = std::sqrt(f.tN / 2.0);
        }
        f.keyLo = k0;
        f.keyHi = k1;
        if (precision == DSMC_PRECISION_MIXED) launch_fill<float>(args<float>(), f, placeFirst, shape, stream);
        else launch_fill<double>(args<double>(), f, placeFirst, shape, stream);
        if (!cuda(cudaGetLastError(), "fill kernel")) return false;
        StepCtl h{};
        h.nLive = (int)total;
        h.capacity = (int)capacity;
        if (!cuda(cudaMemcpyAsync(ctl, &h, sizeof h, cudaMemcpyHostToDevice, stream), "ctl")) return false;
        if (!cuda(cudaMemsetAsync(countSlot, 0, (size_t)ncell * kSlots * sizeof(int), stream), "countSlot")) return false;
        if (!cuda(cudaStreamSynchronize(stream), "fill sync")) return false;
        hostNLive = (int)total;
        haveParticles = true;
        devIstepValid = false;
        pendingInject = false;
        return true;
    }

    // GSIS particle update (molecular_velocity_change, src/ProcessGSIS.cpp:
    // 2239-2366) between steps; see csrc/dsmc_gsis.cu.
    bool gsisUpdate(const double* ns, const char* accepted, DsmcGsisReport* rep)
    {
        if (!ns) return fail("GSIS: null nsresult");
        if (!haveParticles) return fail("GSIS: no particles");
        if (pendingInject) return fail("GSIS: a step is in progress (injected particles not yet sorted)");
        // the reference stops at the first gated-in cell with a NaN density or velocity
        int firstNan = ncell;
        for (int c = 0; c < ncell && firstNan == ncell; ++c) {
            if (accepted && accepted[c] == 0) continue;
            const double* r = ns + (size_t)c * 6;
            if (std::isnan(r[0]) || std::isnan(r[1]) || std::isnan(r[2]) || std::isnan(r[3])) firstNan = c;
        }
        if (!gsisNs && (!alloc(gsisNs, (size_t)ncell * 6, false) || !alloc(gsisAcc, (size_t)ncell, false) ||
                        !alloc(gsisFlag, (size_t)ncell, false) || !alloc(gsisTally, 4, false)))
            return false;
        if (!cuda(cudaMemcpyAsync(gsisNs, ns, (size_t)ncell * 6 * sizeof(double), cudaMemcpyHostToDevice, stream), "GSIS ns") ||
            (accepted && !cuda(cudaMemcpyAsync(gsisAcc, accepted, (size_t)ncell, cudaMemcpyHostToDevice, stream), "GSIS gate")) ||
            !cuda(cudaMemsetAsync(gsisTally, 0, 4 * sizeof(unsigned long long), stream), "GSIS tally"))
            return false;
        GsisArgs g{};
        g.ns = gsisNs;
        g.accepted = accepted ? gsisAcc : nullptr;
        g.firstNan = firstNan;
        g.keyLo = C.seedLo;
        g.keyHi = C.seedHi;
        g.purpose = kPurposeGsis | ((gsisEpoch & 0xffffffu) << 8);
        g.flag = gsisFlag;
        g.tally = gsisTally;
        int err0 = 0;
        if (!cuda(cudaMemcpyAsync(&err0, errorWord, sizeof(int), cudaMemcpyDeviceToHost, stream), "error word"))
            return false;
        if (precision == DSMC_PRECISION_MIXED) launch_gsis_count<float>(args<float>(), g, stream);
        else launch_gsis_count<double>(args<double>(), g, stream);
        if (!cuda(cudaGetLastError(), "GSIS count")) return false;
        StepCtl h{};
        int err1 = 0;
        if (!cuda(cudaMemcpyAsync(&h, ctl, sizeof h, cudaMemcpyDeviceToHost, stream), "ctl") ||
            !cuda(cudaMemcpyAsync(&err1, errorWord, sizeof(int), cudaMemcpyDeviceToHost, stream), "error word") ||
            !cuda(cudaStreamSynchronize(stream), "GSIS count sync"))
            return false;
        auto abandon = [&](const std::string& m) {
            cudaMemcpyAsync(errorWord, &err0, sizeof(int), cudaMemcpyHostToDevice, stream);
            cudaMemsetAsync(countSlot, 0, (size_t)ncell * kSlots * sizeof(int), stream);
            cudaStreamSynchronize(stream);
            return fail(m);
        };
        if ((err1 & ~err0) & kErrGsisCount)
            return abandon("GSIS: an NS density gives a particle count outside [0, 2^30)");
        const int64_t nNext = h.nNext;
        if (nNext > capacity) {
            if (params.capacity > 0) return abandon("GSIS: more particles than the configured capacity");
            // growing keeps the particles of A; the counts and the layout of B stay valid
            if (!ensureCapacity(std::max<int64_t>(nNext + nNext / 2 + (1 << 16), 1 << 20))) return false;
        }
        if (precision == DSMC_PRECISION_MIXED) launch_gsis_rebuild<float>(args<float>(), g, shape, stream);
        else launch_gsis_rebuild<double>(args<double>(), g, shape, stream);
        if (!cuda(cudaGetLastError(), "GSIS rebuild")) return false;
        cur ^= 1;
        h.nLive = (int)nNext;
        h.nInj = 0;
        h.capacity = (int)capacity;
        unsigned long long tally[4] = {0, 0, 0, 0};
        if (!cuda(cudaMemcpyAsync(ctl, &h, sizeof h, cudaMemcpyHostToDevice, stream), "ctl") ||
            !cuda(cudaMemsetAsync(countSlot, 0, (size_t)ncell * kSlots * sizeof(int), stream), "countSlot") ||
            !cuda(cudaMemcpyAsync(tally, gsisTally, sizeof tally, cudaMemcpyDeviceToHost, stream), "GSIS tally") ||
            !cuda(cudaStreamSynchronize(stream), "GSIS sync"))
            return false;
        hostNLive = (int)nNext;
        devIstepValid = false;
        ++gsisEpoch;
        if (rep) {
            rep->nan_cell = firstNan < ncell ? firstNan : -1;
            rep->cells_updated = (int32_t)tally[0];
            rep->cells_skipped = (int32_t)tally[1];
            rep->added = (int64_t)tally[2];
            rep->removed = (int64_t)tally[3];
            rep->particles = nNext;
        }
        return true;
    }

    bool downloadParticles(int64_t n, double* px, double* py, double* pz, double* vx, double* vy, double* vz,
                           double* ir, int32_t* cellOut, uint32_t* pid)
    {
        int nl = 0;
        if (!nLiveHost(nl)) return false;
        if (n != nl) return fail("particle count mismatch: call dsmc_particle_count first");
        std::vector<int> hc((size_t)n);
        if (n > 0 && !cuda(cudaMemcpy(hc.data(), buf[cur][7], (size_t)n * sizeof(int), cudaMemcpyDeviceToHost), "cells"))
            return false;
        double* dst[7] = {px, py, pz, vx, vy, vz, ir};
        const bool mixed = precision == DSMC_PRECISION_MIXED;
        std::vector<char> hb((size_t)n * 8);
        const int nthreads = hostpack::threads_for(n);
        for (int k = 0; k < 7; ++k) {
            if (!dst[k] || n == 0) continue;
            if (!cuda(cudaMemcpy(hb.data(), buf[cur][k], (size_t)n * realSize(), cudaMemcpyDeviceToHost), "particles"))
                return false;
            if (mixed)
                hostpack::widen<float>(n, reinterpret_cast<const float*>(hb.data()), hc.data(),
                                       k < 3 ? cellCenterHost.data() : nullptr, k, dst[k], nthreads);
            else
                hostpack::widen<double>(n, reinterpret_cast<const double*>(hb.data()), hc.data(), nullptr, k, dst[k],
                                        nthreads);
        }
        if (cellOut) std::memcpy(cellOut, hc.data(), (size_t)n * sizeof(int));
        if (pid) for (int64_t j = 0; j < n; ++j) pid[j] = (uint32_t)j;
        return true;
    }

    bool downloadMacro(int which, double* out)
    {
        if (!out) return fail("null output");
        double* src = nullptr;
        if (which == DSMC_MACRO_LOCAL) {
            if (localLazy) launch_macro(M, C, acc, 0, (double)params.nscheme, local, ncell, stream);
            src = local;
        } else if (which == DSMC_MACRO_RECORD) {
            src = record;
        } else if (which == DSMC_MACRO_FINAL_RECORD) {
            if (lastIstep > params.nss)
                launch_macro(M, C, acc, 1, (double)(lastIstep - params.nss), finalRecord, ncell, stream);
            src = finalRecord;
        } else {
            return fail("unknown macro target");
        }
        if (!cuda(cudaMemcpyAsync(out, src, (size_t)ncell * 18 * sizeof(double), cudaMemcpyDeviceToHost, stream), "macro"))
            return false;
        return cuda(cudaStreamSynchronize(stream), "macro sync");
    }
};

}  // namespace dsmc

struct DsmcHandle {
    dsmc::Engine e;
};

static thread_local std::string g_createError;

#define DSMC_GUARD(h)                                                   \
    do {                                                                \
        if (!(h)) return DSMC_E_INVALID;                                \
        if ((h)->e.device >= 0) cudaSetDevice((h)->e.device);           \
    } while (0)

// No C++ exception crosses the C ABI: the entry points that allocate on the
// host are function-try-blocks ending in DSMC_CATCH(err), which turns an
// exception into a status and a message in *err (the handle's, the batch's,
// or the create error).
static int host_exception(std::string* err, int code, const char* what) noexcept
{
    if (err) {
        try {
            *err = what;
        } catch (...) {
        }
    }
    return code;
}

#define DSMC_CATCH(err)                                                                              \
    catch (const std::bad_alloc&) { return host_exception((err), DSMC_E_NOMEM, "host allocation failed"); }  \
    catch (const std::length_error&) { return host_exception((err), DSMC_E_NOMEM, "host allocation failed"); } \
    catch (const std::exception& ex) { return host_exception((err), DSMC_E_INVALID, ex.what()); }            \
    catch (...) { return host_exception((err), DSMC_E_INVALID, "host exception"); }

static int status_of(dsmc::Engine& e, bool ok)
{
    if (ok) return DSMC_OK;
    if (e.err.find("cudaMalloc") != std::string::npos) return DSMC_E_NOMEM;
    if (e.err.find("capacity") != std::string::npos) return DSMC_E_CAPACITY;
    if (e.err.find(": ") != std::string::npos && e.err.find("cuda") != std::string::npos) return DSMC_E_CUDA;
    if (e.err.find("rejection loop") != std::string::npos) return DSMC_E_DEVICE_FAULT;
    if (e.err.find("self-check") != std::string::npos) return DSMC_E_DEVICE_FAULT;
    if (e.err.find("no particles") != std::string::npos) return DSMC_E_STATE;
    if (e.err.find("in progress") != std::string::npos) return DSMC_E_STATE;
    return DSMC_E_INVALID;
}

extern "C" {

void dsmc_default_params(DsmcCaseParams* p)
{
    if (!p) return;
    std::memset(p, 0, sizeof(*p));
    p->precision = DSMC_PRECISION_FP64;
    p->nss = 5000;       // src/meshImport.h:48
    p->nscheme = 2000;   // src/meshImport.h:56
    p->nevery = 1;       // src/meshImport.h:52
    p->nrepeat = 100;    // src/meshImport.h:53
    p->wall_stats = 0;   // src/meshImport.h:50
    p->inflow_dir[0] = std::sqrt(3.0) / 2.0;   // src/ProcessDSMC.cpp:2330-2331
    p->inflow_dir[1] = 0.5;
    // BoundaryConditionTable::loadDefaults, src/BoundaryCondition.h:79-117
    p->nzones = 4;
    p->zone_tag[0] = 3; p->zone_role[0] = DSMC_ROLE_INTERFACE; p->zone_inject[0] = 0;
    p->zone_tag[1] = 4; p->zone_role[1] = DSMC_ROLE_INLET; p->zone_inject[1] = 1;
    p->zone_tag[2] = 5; p->zone_role[2] = DSMC_ROLE_OUTLET; p->zone_inject[2] = 0;
    p->zone_tag[3] = 6; p->zone_role[3] = DSMC_ROLE_WALL; p->zone_inject[3] = 0;
    p->capacity = 0;
    p->seed = 0;
    p->max_crossings = 4096;
    p->keep_step_moments = 0;
}

int dsmc_create(const DsmcMeshDesc* mesh, const DsmcMeshMessage* mess, const DsmcCaseParams* params, int device,
                DsmcHandle** out)
try {
    if (!out) return DSMC_E_INVALID;
    *out = nullptr;
    std::unique_ptr<DsmcHandle> h(new (std::nothrow) DsmcHandle());
    if (!h) return DSMC_E_NOMEM;
    if (!h->e.build(mesh, mess, params, device)) {
        g_createError = h->e.err;
        return status_of(h->e, false);
    }
    *out = h.release();
    return DSMC_OK;
}
DSMC_CATCH(&g_createError)

void dsmc_destroy(DsmcHandle* h) { delete h; }

const char* dsmc_last_error(const DsmcHandle* h) { return h ? h->e.err.c_str() : g_createError.c_str(); }

int dsmc_upload_particles(DsmcHandle* h, int64_t n, const double* px, const double* py, const double* pz,
                          const double* vx, const double* vy, const double* vz, const double* ir, const int32_t* cell)
try {
    DSMC_GUARD(h);
    return status_of(h->e, h->e.uploadParticles(n, px, py, pz, vx, vy, vz, ir, cell));
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_particle_count(DsmcHandle* h, int64_t* n)
{
    DSMC_GUARD(h);
    if (!n) return DSMC_E_INVALID;
    int nl = 0;
    if (!h->e.haveParticles) { *n = 0; return DSMC_OK; }
    const bool ok = h->e.nLiveHost(nl);
    *n = nl;
    return status_of(h->e, ok);
}

int dsmc_download_particles(DsmcHandle* h, int64_t n, double* px, double* py, double* pz, double* vx, double* vy,
                            double* vz, double* ir, int32_t* cell, uint32_t* pid)
try {
    DSMC_GUARD(h);
    if (!h->e.haveParticles) return n == 0 ? DSMC_OK : DSMC_E_STATE;
    return status_of(h->e, h->e.downloadParticles(n, px, py, pz, vx, vy, vz, ir, cell, pid));
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_step(DsmcHandle* h, int32_t istep, uint32_t stages)
try {
    DSMC_GUARD(h);
    return status_of(h->e, h->e.step(istep, stages));
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_preprocesseffquad(DsmcHandle* h, int32_t istep) { return dsmc_step(h, istep, DSMC_STAGE_INJECT); }
int dsmc_advection(DsmcHandle* h, int32_t istep) { return dsmc_step(h, istep, DSMC_STAGE_MOVE); }
int dsmc_cache2chain(DsmcHandle* h)
{
    DSMC_GUARD(h);
    return status_of(h->e, h->e.step(h->e.curIstep, DSMC_STAGE_SORT));
}
int dsmc_collisionDSMC(DsmcHandle* h)
{
    DSMC_GUARD(h);
    // the collision stream is keyed by the step of the preceding stage calls
    return status_of(h->e, h->e.step(h->e.curIstep, DSMC_STAGE_COLLIDE));
}
int dsmc_statistic_macro(DsmcHandle* h, int32_t istep) { return dsmc_step(h, istep, DSMC_STAGE_SAMPLE); }
int dsmc_statistic_macroPre(DsmcHandle* h)
{
    DSMC_GUARD(h);
    return status_of(h->e, h->e.macroPre());
}

int dsmc_download_macro(DsmcHandle* h, int32_t which, double* out)
{
    DSMC_GUARD(h);
    return status_of(h->e, h->e.downloadMacro(which, out));
}

int dsmc_download_counts(DsmcHandle* h, int32_t* ppc, double* window_samples, char* window_valid,
                         unsigned char* sparse_state, double* stepinter_rho, double* steady_rho)
try {
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    const size_t nc = (size_t)e.ncell;
    bool ok = true;
    if (ppc) {
        std::vector<int> st(nc + 1, 0);
        if (e.haveParticles)
            ok = ok && e.cuda(cudaMemcpyAsync(st.data(), e.start[e.cur], (nc + 1) * sizeof(int), cudaMemcpyDeviceToHost, e.stream), "start");
        ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
        for (size_t c = 0; c < nc && ok; ++c) ppc[c] = st[c + 1] - st[c];
    }
    if (ok && window_samples) ok = e.cuda(cudaMemcpyAsync(window_samples, e.windowSamples, nc * sizeof(double), cudaMemcpyDeviceToHost, e.stream), "ws");
    if (ok && window_valid) ok = e.cuda(cudaMemcpyAsync(window_valid, e.windowValid, nc, cudaMemcpyDeviceToHost, e.stream), "wv");
    if (ok && sparse_state) ok = e.cuda(cudaMemcpyAsync(sparse_state, e.sparseState, nc, cudaMemcpyDeviceToHost, e.stream), "ss");
    if (ok && stepinter_rho)
        ok = e.cuda(cudaMemcpy2DAsync(stepinter_rho, sizeof(double), e.acc + 36, 54 * sizeof(double), sizeof(double), nc,
                                      cudaMemcpyDeviceToHost, e.stream), "stepinter");
    if (ok && steady_rho)
        ok = e.cuda(cudaMemcpy2DAsync(steady_rho, sizeof(double), e.acc + 18, 54 * sizeof(double), sizeof(double), nc,
                                      cudaMemcpyDeviceToHost, e.stream), "steady");
    ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
    return status_of(e, ok);
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_download_step_moments(DsmcHandle* h, double* out)
{
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    if (!e.stepMom) { e.err = "step moments not kept (params.keep_step_moments)"; return DSMC_E_STATE; }
    bool ok = e.cuda(cudaMemcpyAsync(out, e.stepMom, (size_t)e.ncell * 18 * sizeof(double), cudaMemcpyDeviceToHost, e.stream), "moments");
    ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
    return status_of(e, ok);
}

int dsmc_download_wall(DsmcHandle* h, double* tally)
try {
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    if (!tally) return DSMC_E_INVALID;
    std::vector<double> w((size_t)std::max(e.nwall, 1) * 6);
    bool ok = e.cuda(cudaMemcpyAsync(w.data(), e.wallTally, w.size() * sizeof(double), cudaMemcpyDeviceToHost, e.stream), "wall");
    ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
    if (!ok) return status_of(e, false);
    std::memset(tally, 0, (size_t)e.nface * 6 * sizeof(double));
    for (int f = 0; f < e.nface; ++f) {
        const int s = e.faceWallHost[(size_t)f];
        if (s >= 0 && e.faceRole[(size_t)f] == DSMC_ROLE_WALL)
            for (int k = 0; k < 6; ++k) tally[(size_t)f * 6 + k] = w[(size_t)s * 6 + k];
    }
    return DSMC_OK;
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_download_cell_state(DsmcHandle* h, double* crmax, double* rem_coll, double* rem_inj)
{
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    const size_t b = (size_t)e.ncell * sizeof(double);
    bool ok = true;
    if (crmax) ok = ok && e.cuda(cudaMemcpyAsync(crmax, e.crmax, b, cudaMemcpyDeviceToHost, e.stream), "crmax");
    if (rem_coll) ok = ok && e.cuda(cudaMemcpyAsync(rem_coll, e.remColl, b, cudaMemcpyDeviceToHost, e.stream), "remcoll");
    if (rem_inj) ok = ok && e.cuda(cudaMemcpyAsync(rem_inj, e.remInj, b, cudaMemcpyDeviceToHost, e.stream), "reminj");
    ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
    return status_of(e, ok);
}

int dsmc_upload_cell_state(DsmcHandle* h, const double* crmax, const double* rem_coll, const double* rem_inj)
{
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    const size_t b = (size_t)e.ncell * sizeof(double);
    bool ok = true;
    if (crmax) ok = ok && e.cuda(cudaMemcpyAsync(e.crmax, crmax, b, cudaMemcpyHostToDevice, e.stream), "crmax");
    if (rem_coll) ok = ok && e.cuda(cudaMemcpyAsync(e.remColl, rem_coll, b, cudaMemcpyHostToDevice, e.stream), "remcoll");
    if (rem_inj) ok = ok && e.cuda(cudaMemcpyAsync(e.remInj, rem_inj, b, cudaMemcpyHostToDevice, e.stream), "reminj");
    ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
    return status_of(e, ok);
}

int dsmc_upload_sparse_state(DsmcHandle* h, const unsigned char* sparse_state)
{
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    if (!sparse_state) return DSMC_E_INVALID;
    for (int c = 0; c < e.ncell; ++c)
        if (sparse_state[c] > 2) {
            e.err = "sparse state outside 0..2";
            return DSMC_E_INVALID;
        }
    bool ok = e.cuda(cudaMemcpyAsync(e.sparseState, sparse_state, (size_t)e.ncell, cudaMemcpyHostToDevice, e.stream),
                     "sparse state");
    ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
    return status_of(e, ok);
}

int dsmc_get_counters(DsmcHandle* h, DsmcCounters* out)
{
    DSMC_GUARD(h);
    if (!out) return DSMC_E_INVALID;
    dsmc::Engine& e = h->e;
    unsigned long long c[dsmc::C_COUNT];
    bool ok = e.cuda(cudaMemcpyAsync(c, e.counters, sizeof c, cudaMemcpyDeviceToHost, e.stream), "counters");
    ok = ok && e.cuda(cudaStreamSynchronize(e.stream), "sync");
    if (!ok) return status_of(e, false);
    out->steps = e.steps;
    out->injected = c[dsmc::C_INJECTED];
    out->removed = c[dsmc::C_REMOVED];
    out->dropped = c[dsmc::C_DROPPED];
    out->lost = c[dsmc::C_LOST];
    out->wall_hits = c[dsmc::C_WALL_HITS];
    out->crossings = c[dsmc::C_CROSSINGS];
    out->candidate_pairs = c[dsmc::C_PAIRS];
    out->collisions = c[dsmc::C_COLLISIONS];
    out->fp64_fallbacks = c[dsmc::C_FALLBACKS];
    out->overflow = c[dsmc::C_OVERFLOW];
    out->big_cells = c[dsmc::C_BIG_CELLS];
    return DSMC_OK;
}

int dsmc_trace(DsmcHandle* h, int64_t n, const double* px, const double* py, const double* pz, const double* vx,
               const double* vy, const double* vz, const double* dt, const int32_t* cell, int32_t stop_at_wall,
               int32_t* out_cell, int32_t* out_ifout, int32_t* out_face, int32_t* out_tri, int32_t* out_ncross,
               double* out_px, double* out_py, double* out_pz, double* out_vx, double* out_vy, double* out_vz,
               double* out_dt)
try {
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    if (n < 0 || n > 0x7fffffff) return DSMC_E_INVALID;
    if (n == 0) return DSMC_OK;
    if (!px || !py || !pz || !vx || !vy || !vz || !dt || !cell) return DSMC_E_INVALID;
    for (int64_t i = 0; i < n; ++i)
        if (cell[i] < 0 || cell[i] >= e.ncell) { e.err = "trace: cell id out of range"; return DSMC_E_INVALID; }
    const bool mixed = e.precision == DSMC_PRECISION_MIXED;
    const size_t rs = mixed ? 4 : 8;
    // device scratch of this call: every failed allocation is recorded, and
    // whatever was allocated is freed on every way out
    struct DeviceTemps {
        std::vector<void*> ptrs;
        bool failed = false;
        void* alloc(size_t bytes)
        {
            ptrs.reserve(ptrs.size() + 1);
            void* q = nullptr;
            if (cudaMalloc(&q, std::max<size_t>(bytes, 1)) != cudaSuccess) {
                failed = true;
                (void)cudaGetLastError();
                return nullptr;
            }
            ptrs.push_back(q);
            return q;
        }
        ~DeviceTemps()
        {
            for (void* q : ptrs) cudaFree(q);
        }
    } tmp;
    auto dal = [&](size_t bytes) -> void* { return tmp.alloc(bytes); };
    void* dIn[6];
    void* dOut[6];
    for (int k = 0; k < 6; ++k) {
        dIn[k] = dal((size_t)n * rs);
        dOut[k] = dal((size_t)n * rs);
    }
    double* dDt = (double*)dal((size_t)n * 8);
    double* dODt = (double*)dal((size_t)n * 8);
    int* dCell = (int*)dal((size_t)n * 4);
    int* dI[6];
    for (int k = 0; k < 6; ++k) dI[k] = (int*)dal((size_t)n * 4);
    if (tmp.failed) { e.err = "trace: device allocation failed"; return DSMC_E_NOMEM; }
    const double* src[6] = {px, py, pz, vx, vy, vz};
    std::vector<char> hb((size_t)n * 8);
    bool ok = true;
    for (int k = 0; k < 6 && ok; ++k) {
        for (int64_t i = 0; i < n; ++i) {
            double v = src[k][i];
            if (mixed) {
                if (k < 3) v -= e.cellCenterHost[(size_t)cell[i] * 3 + k];
                reinterpret_cast<float*>(hb.data())[i] = (float)v;
            } else {
                reinterpret_cast<double*>(hb.data())[i] = v;
            }
        }
        ok = e.cuda(cudaMemcpy(dIn[k], hb.data(), (size_t)n * rs, cudaMemcpyHostToDevice), "trace upload");
    }
    ok = ok && e.cuda(cudaMemcpy(dDt, dt, (size_t)n * 8, cudaMemcpyHostToDevice), "trace dt");
    ok = ok && e.cuda(cudaMemcpy(dCell, cell, (size_t)n * 4, cudaMemcpyHostToDevice), "trace cells");
    if (ok) {
        if (mixed)
            dsmc::launch_trace_check<float>(e.M, e.C, (int)n, (float*)dIn[0], (float*)dIn[1], (float*)dIn[2],
                                            (float*)dIn[3], (float*)dIn[4], (float*)dIn[5], dDt, dCell, stop_at_wall,
                                            dI[0], dI[1], dI[2], dI[3], dI[4], dI[5], (float*)dOut[0], (float*)dOut[1],
                                            (float*)dOut[2], (float*)dOut[3], (float*)dOut[4], (float*)dOut[5], dODt,
                                            e.counters, e.stream);
        else
            dsmc::launch_trace_check<double>(e.M, e.C, (int)n, (double*)dIn[0], (double*)dIn[1], (double*)dIn[2],
                                             (double*)dIn[3], (double*)dIn[4], (double*)dIn[5], dDt, dCell,
                                             stop_at_wall, dI[0], dI[1], dI[2], dI[3], dI[4], dI[5], (double*)dOut[0],
                                             (double*)dOut[1], (double*)dOut[2], (double*)dOut[3], (double*)dOut[4],
                                             (double*)dOut[5], dODt, e.counters, e.stream);
        ok = e.cuda(cudaGetLastError(), "trace launch") && e.cuda(cudaStreamSynchronize(e.stream), "trace sync");
    }
    std::vector<int> last((size_t)n);
    int32_t* iout[5] = {out_cell, out_ifout, out_face, out_tri, out_ncross};
    for (int k = 0; k < 5 && ok; ++k)
        if (iout[k]) ok = e.cuda(cudaMemcpy(iout[k], dI[k], (size_t)n * 4, cudaMemcpyDeviceToHost), "trace out");
    ok = ok && e.cuda(cudaMemcpy(last.data(), dI[5], (size_t)n * 4, cudaMemcpyDeviceToHost), "trace last");
    double* fout[6] = {out_px, out_py, out_pz, out_vx, out_vy, out_vz};
    for (int k = 0; k < 6 && ok; ++k) {
        if (!fout[k]) continue;
        ok = e.cuda(cudaMemcpy(hb.data(), dOut[k], (size_t)n * rs, cudaMemcpyDeviceToHost), "trace out");
        for (int64_t i = 0; i < n && ok; ++i) {
            double v = mixed ? (double)reinterpret_cast<float*>(hb.data())[i] : reinterpret_cast<double*>(hb.data())[i];
            if (mixed && k < 3) v = e.cellCenterHost[(size_t)last[(size_t)i] * 3 + k] + v;
            fout[k][i] = v;
        }
    }
    if (ok && out_dt) ok = e.cuda(cudaMemcpy(out_dt, dODt, (size_t)n * 8, cudaMemcpyDeviceToHost), "trace dt out");
    return status_of(e, ok);
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_set_timing(DsmcHandle* h, int32_t on)
{
    DSMC_GUARD(h);
    h->e.timing = on != 0;
    return DSMC_OK;
}

int dsmc_stage_ms(DsmcHandle* h, double* ms5, int64_t* nsteps, int32_t reset)
{
    DSMC_GUARD(h);
    if (ms5)
        for (int k = 0; k < 5; ++k) ms5[k] = h->e.stageMs[k];
    if (nsteps) *nsteps = h->e.timedSteps;
    if (reset) {
        for (double& v : h->e.stageMs) v = 0.0;
        h->e.timedSteps = 0;
    }
    return DSMC_OK;
}

void* dsmc_stream(DsmcHandle* h) { return h ? (void*)h->e.stream : nullptr; }

int dsmc_sync(DsmcHandle* h)
{
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    bool ok = e.cuda(cudaStreamSynchronize(e.stream), "sync") && e.checkDeviceErrors();
    return status_of(e, ok);
}


// Read-only views of a handle for the no-allocation entry point
// (dsmc_noalloc.cu).
}  // extern "C"

namespace dsmc {
DevMesh engine_mesh(const DsmcHandle* h) { return h->e.M; }
DevConsts engine_consts(const DsmcHandle* h) { return h->e.C; }
int engine_precision(const DsmcHandle* h) { return h->e.precision; }
int engine_device(const DsmcHandle* h) { return h->e.device; }
cudaStream_t engine_stream(const DsmcHandle* h) { return h->e.stream; }
unsigned long long* engine_counters(const DsmcHandle* h) { return h->e.counters; }
// Sets the handle's message; a failed host allocation leaves the previous
// one (nothing is thrown across the C ABI).
void engine_set_error(DsmcHandle* h, const char* msg) noexcept
{
    try {
        h->e.err = msg;
    } catch (...) {
    }
}
}  // namespace dsmc

extern "C" {

int dsmc_fill_freestream(DsmcHandle* h, double ppc_mean, uint64_t seed)
try {
    DSMC_GUARD(h);
    return status_of(h->e, h->e.fill(ppc_mean, seed, false));
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_fill_initial(DsmcHandle* h, double ppc_mean, uint64_t seed)
try {
    DSMC_GUARD(h);
    return status_of(h->e, h->e.fill(ppc_mean, seed, true));
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_molecular_velocity_change(DsmcHandle* h, const double* nsresult, const char* accepted,
                                   DsmcGsisReport* report)
try {
    DSMC_GUARD(h);
    return status_of(h->e, h->e.gsisUpdate(nsresult, accepted, report));
}
DSMC_CATCH(h ? &h->e.err : nullptr)

// ---------------------------------------------------------------------------
// launch shapes and the autotuner
// ---------------------------------------------------------------------------
int dsmc_get_launch_shape(DsmcHandle* h, DsmcLaunchShape* out)
{
    DSMC_GUARD(h);
    if (!out) return DSMC_E_INVALID;
    *out = h->e.getShape();
    return DSMC_OK;
}

int dsmc_set_launch_shape(DsmcHandle* h, const DsmcLaunchShape* shape)
try {
    DSMC_GUARD(h);
    if (!shape) return DSMC_E_INVALID;
    return h->e.setShape(*shape) ? DSMC_OK : DSMC_E_INVALID;
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_autotune(DsmcHandle* h, int32_t first_istep, int32_t trial_steps, int32_t* next_istep,
                  DsmcLaunchShape* chosen)
try {
    DSMC_GUARD(h);
    int istep = first_istep;
    const bool ok = h->e.autotune(istep, trial_steps);
    if (next_istep) *next_istep = istep;
    if (chosen) *chosen = h->e.getShape();
    return status_of(h->e, ok);
}
DSMC_CATCH(h ? &h->e.err : nullptr)

// ---------------------------------------------------------------------------
// batched steps
// ---------------------------------------------------------------------------
struct DsmcBatch {
    std::vector<DsmcHandle*> cases;
    int device = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t fork = nullptr;
    cudaEvent_t done = nullptr;
    std::vector<cudaEvent_t> join;
    struct Cached {
        std::vector<int> key;
        cudaGraphExec_t exec = nullptr;
    };
    std::vector<Cached> graphs;
    std::string err;

    ~DsmcBatch()
    {
        cudaSetDevice(device);
        if (stream) cudaStreamSynchronize(stream);
        for (auto& g : graphs)
            if (g.exec) cudaGraphExecDestroy(g.exec);
        for (auto e : join)
            if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (done) cudaEventDestroy(done);
        if (stream) cudaStreamDestroy(stream);
    }
    bool fail(const std::string& m)
    {
        err = m;
        return false;
    }
    bool cuda(cudaError_t e, const char* what)
    {
        if (e == cudaSuccess) return true;
        return fail(std::string(what) + ": " + cudaGetErrorString(e));
    }
    // the graph state of every case: buffer parity and graph generation
    std::vector<int> key() const
    {
        std::vector<int> k;
        k.reserve(cases.size() * 2);
        for (DsmcHandle* h : cases) {
            k.push_back(h->e.cur);
            k.push_back(h->e.generation);
        }
        return k;
    }
    bool capture(cudaGraphExec_t& exec)
    {
        cudaGraph_t g = nullptr;
        if (!cuda(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal), "batch capture")) return false;
        cudaEventRecord(fork, stream);
        for (size_t k = 0; k < cases.size(); ++k) {
            dsmc::Engine& e = cases[k]->e;
            cudaStreamWaitEvent(e.stream, fork, 0);
            e.enqueueBatch();
            cudaEventRecord(join[k], e.stream);
            cudaStreamWaitEvent(stream, join[k], 0);
        }
        if (!cuda(cudaStreamEndCapture(stream, &g), "batch end capture")) return false;
        const cudaError_t ie = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        return cuda(ie, "batch graph instantiate");
    }
    bool step(int nsteps)
    {
        if (nsteps < 0) return fail("negative step count");
        if (nsteps == 0) return true;
        for (DsmcHandle* h : cases) {
            dsmc::Engine& e = h->e;
            if (!e.haveParticles) return fail("a case of the batch has no particles");
            if (e.timing) return fail("a case of the batch is in timing mode");
            if (!e.devIstepValid) {
                if (!e.setIstep(e.curIstep)) return fail("istep: " + e.err);
                e.devIstepValid = true;
            }
            // the batch stream starts after the work already queued on each case
            cudaEventRecord(done, e.stream);
            cudaStreamWaitEvent(stream, done, 0);
        }
        for (int s = 0; s < nsteps; ++s) {
            const std::vector<int> k = key();
            cudaGraphExec_t exec = nullptr;
            for (auto& c : graphs)
                if (c.key == k) exec = c.exec;
            if (!exec) {
                if (graphs.size() >= 4) {   // stale entries (a case was re-uploaded)
                    cudaStreamSynchronize(stream);
                    cudaGraphExecDestroy(graphs.front().exec);
                    graphs.erase(graphs.begin());
                }
                if (!capture(exec)) return false;
                graphs.push_back(Cached{k, exec});
            }
            if (!cuda(cudaGraphLaunch(exec, stream), "batch graph launch")) return false;
            for (DsmcHandle* h : cases) h->e.afterBatchStep();
        }
        // later work on each case's own stream follows the batch
        cudaEventRecord(done, stream);
        for (DsmcHandle* h : cases) cudaStreamWaitEvent(h->e.stream, done, 0);
        return cuda(cudaGetLastError(), "batch step");
    }
};

int dsmc_batch_create(DsmcHandle* const* cases, int32_t n, DsmcBatch** out)
try {
    if (!out) return DSMC_E_INVALID;
    *out = nullptr;
    if (!cases || n < 1) {
        g_createError = "dsmc_batch_create: no cases";
        return DSMC_E_INVALID;
    }
    for (int32_t k = 0; k < n; ++k) {
        if (!cases[k]) {
            g_createError = "dsmc_batch_create: null case handle";
            return DSMC_E_INVALID;
        }
        if (cases[k]->e.device != cases[0]->e.device) {
            g_createError = "dsmc_batch_create: cases on different devices";
            return DSMC_E_INVALID;
        }
        for (int32_t j = 0; j < k; ++j)
            if (cases[j] == cases[k]) {
                g_createError = "dsmc_batch_create: a case appears twice";
                return DSMC_E_INVALID;
            }
    }
    std::unique_ptr<DsmcBatch> b(new (std::nothrow) DsmcBatch());
    if (!b) return DSMC_E_NOMEM;
    b->cases.assign(cases, cases + n);
    b->device = cases[0]->e.device;
    cudaSetDevice(b->device);
    bool ok = b->cuda(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking), "batch stream") &&
              b->cuda(cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming), "batch event") &&
              b->cuda(cudaEventCreateWithFlags(&b->done, cudaEventDisableTiming), "batch event");
    b->join.assign((size_t)n, nullptr);
    for (int32_t k = 0; ok && k < n; ++k)
        ok = b->cuda(cudaEventCreateWithFlags(&b->join[(size_t)k], cudaEventDisableTiming), "batch event");
    if (!ok) {
        g_createError = b->err;
        return DSMC_E_CUDA;
    }
    *out = b.release();
    return DSMC_OK;
}
DSMC_CATCH(&g_createError)

void dsmc_batch_destroy(DsmcBatch* b) { delete b; }

const char* dsmc_batch_last_error(const DsmcBatch* b) { return b ? b->err.c_str() : g_createError.c_str(); }

int dsmc_batch_step(DsmcBatch* b, int32_t nsteps)
try {
    if (!b) return DSMC_E_INVALID;
    cudaSetDevice(b->device);
    return b->step(nsteps) ? DSMC_OK : DSMC_E_STATE;
}
DSMC_CATCH(b ? &b->err : nullptr)

void* dsmc_batch_stream(DsmcBatch* b) { return b ? (void*)b->stream : nullptr; }

int dsmc_batch_sync(DsmcBatch* b)
{
    if (!b) return DSMC_E_INVALID;
    cudaSetDevice(b->device);
    if (!b->cuda(cudaStreamSynchronize(b->stream), "batch sync")) return DSMC_E_CUDA;
    for (DsmcHandle* h : b->cases)
        if (!h->e.checkDeviceErrors()) return b->fail(h->e.err), status_of(h->e, false);
    return DSMC_OK;
}


// ---------------------------------------------------------------------------
// field output (ProcessDSMC::out2dat, outBoundaryStressHeat)
// ---------------------------------------------------------------------------
int dsmc_out2dat(DsmcHandle* h, int32_t istep, const DsmcZone* zones, int32_t nzones, const char* path)
try {
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    const size_t nc = (size_t)e.ncell;
    std::vector<double> rec(nc * 18), fin(nc * 18);
    std::vector<unsigned char> sparse(nc, 0);
    if (!e.downloadMacro(DSMC_MACRO_RECORD, rec.data()) || !e.downloadMacro(DSMC_MACRO_FINAL_RECORD, fin.data()))
        return status_of(e, false);
    bool ok = e.cuda(cudaMemcpyAsync(sparse.data(), e.sparseState, nc, cudaMemcpyDeviceToHost, e.stream), "sparse") &&
              e.cuda(cudaStreamSynchronize(e.stream), "sync");
    if (!ok) return status_of(e, false);
    // record up to NSS and for sparse cells (DSMC2NS_SPARSE_ACCUMULATING /
    // RELEASED), final_record after (src/ProcessDSMC.cpp:3346-3364)
    for (size_t c = 0; c < nc; ++c) {
        const bool useRecord = istep <= e.params.nss || sparse[c] == 1 || sparse[c] == 2;
        if (!useRecord) std::memcpy(&rec[c * 18], &fin[c * 18], 18 * sizeof(double));
    }
    const int st = dsmc_write_fluent_cells(path, &e.mess, zones, nzones, rec.data(), e.ncell);
    if (st != DSMC_OK) e.err = dsmc_meshio_last_error();
    return st;
}
DSMC_CATCH(h ? &h->e.err : nullptr)

int dsmc_out_boundary_stress_heat(DsmcHandle* h, int32_t istep, const DsmcZone* zones, int32_t nzones,
                                  const char* path)
try {
    DSMC_GUARD(h);
    dsmc::Engine& e = h->e;
    // EnableBoundaryStressHeatStatistic off: nothing to write
    if (!e.params.wall_stats) return DSMC_OK;
    std::vector<double> tally((size_t)e.nface * 6);
    const int dst = dsmc_download_wall(h, tally.data());
    if (dst != DSMC_OK) return dst;
    const int st = dsmc_write_fluent_wall(path, &e.mess, &e.params, zones, nzones, e.edges.data(), e.nface,
                                          tally.data(), istep);
    if (st != DSMC_OK) e.err = dsmc_meshio_last_error();
    return st;
}
DSMC_CATCH(h ? &h->e.err : nullptr)

}  // extern "C"
