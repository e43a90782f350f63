// Native mesh input and field output: the Fluent ASCII case reader, the DSMC
// topology builder, the case constants and the Fluent data writers
// (include/dsmc_meshio.h). Host code, compiled without fused multiply-add so
// every floating-point operation rounds where the reference's x86-64 build
// rounds it.
#include "dsmc_meshio.h"

#include <algorithm>
#include <cerrno>
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <stdexcept>
#include <string>
#include <vector>

struct DsmcMeshFile {
    std::vector<DsmcCellRec> cells;
    std::vector<DsmcEdgeRec> edges;
    std::vector<double> points;
    std::vector<unsigned char> split;
    std::vector<DsmcZone> zones;
    double areaSum = 0.0;
    double minEdge = 0.0;
    int bcnumber = 0;
};

namespace {

thread_local std::string g_err;

int failWith(const std::string& m, int code = DSMC_E_INVALID)
{
    g_err = m;
    return code;
}

// No C++ exception crosses the C ABI: the entry points that allocate are
// function-try-blocks ending in DSMC_MESHIO_CATCH.
int failNoexcept(const char* m, int code) noexcept
{
    try {
        g_err = m;
    } catch (...) {
    }
    return code;
}

#define DSMC_MESHIO_CATCH                                                                            \
    catch (const std::bad_alloc&) { return failNoexcept("host allocation failed", DSMC_E_NOMEM); }  \
    catch (const std::length_error&) { return failNoexcept("host allocation failed", DSMC_E_NOMEM); } \
    catch (const std::exception& ex) { return failNoexcept(ex.what(), DSMC_E_INVALID); }            \
    catch (...) { return failNoexcept("host exception", DSMC_E_INVALID); }

struct FileCloser {
    void operator()(FILE* f) const
    {
        if (f) std::fclose(f);
    }
};

// ---------------------------------------------------------------------------
// lexing
// ---------------------------------------------------------------------------

// Value of a hexadecimal token, skipping '(' and stopping at ')', as
// meshImport::hex2dcm reads it (src/meshImport.cpp:553-575); upper-case
// digits are accepted too.
long long hexValue(const char* b, const char* e)
{
    long long v = 0;
    for (const char* p = b; p < e; ++p) {
        const char c = *p;
        if (c == ')') break;
        if (c == '(') continue;
        int d;
        if (c >= '0' && c <= '9') d = c - '0';
        else if (c >= 'a' && c <= 'f') d = c - 'a' + 10;
        else if (c >= 'A' && c <= 'F') d = c - 'A' + 10;
        else return -1;
        v = v * 16 + d;
    }
    return v;
}

struct Tok {
    const char* b;
    const char* e;
    bool is(const char* s) const { return (size_t)(e - b) == std::strlen(s) && std::memcmp(b, s, (size_t)(e - b)) == 0; }
    long long hex() const { return hexValue(b, e); }
};

// whitespace-separated tokens of one line
void tokens(const char* b, const char* e, std::vector<Tok>& out)
{
    out.clear();
    const char* p = b;
    while (p < e) {
        while (p < e && (*p == ' ' || *p == '\t' || *p == '\r')) ++p;
        if (p >= e) break;
        const char* q = p;
        while (q < e && *q != ' ' && *q != '\t' && *q != '\r') ++q;
        out.push_back(Tok{p, q});
        p = q;
    }
}

struct Lines {
    const char* p;
    const char* end;
    bool next(const char*& b, const char*& e)
    {
        if (p >= end) return false;
        b = p;
        const char* q = static_cast<const char*>(std::memchr(p, '\n', (size_t)(end - p)));
        e = q ? q : end;
        p = q ? q + 1 : end;
        return true;
    }
};

bool blankOrParen(const char* b, const char* e, size_t minLen)
{
    // "(" alone, or too short to hold data: the lines readNodes / readCells /
    // readFaces skip
    size_t n = (size_t)(e - b);
    while (n > 0 && (b[n - 1] == '\r')) --n;
    return (n == 1 && b[0] == '(') || n <= minLen;
}

// ---------------------------------------------------------------------------
// the raw mesh as the case file gives it
// ---------------------------------------------------------------------------
struct Raw {
    int dim = 3;
    int npoint = 0, ncell = 0, nface = 0;
    std::vector<double> P;          // [npoint*3]
    std::vector<int> cellType;      // [ncell] Fluent element type
    std::vector<int> fnode;         // [nface*4], -1 for the 4th node of a triangle
    std::vector<int> ftype, c0, c1, ftag;
    std::vector<char> fset;         // face given in a data section
    std::vector<DsmcZone> zones;
};

// zone header "(12 (id first last ...)" or "(13 (id first last ...)":
// getZoneid records every declaration whose id is not 0
void zoneHeader(const std::vector<Tok>& t, int section, Raw& r)
{
    if (t.size() < 4 || t[1].is("(0")) return;
    DsmcZone z{};
    z.section = section;
    z.id = (int32_t)t[1].hex();
    z.first = (int32_t)t[2].hex();
    z.last = (int32_t)t[3].hex();
    r.zones.push_back(z);
}

bool parseCas(const char* b, const char* e, Raw& r, std::string& err)
{
    Lines L{b, e};
    const char *lb, *le;
    std::vector<Tok> t, u;
    bool haveNodes = false, haveCells = false, haveFaces = false;
    while (L.next(lb, le)) {
        tokens(lb, le, t);
        if (t.empty()) continue;
        const Tok& s = t[0];
        if (s.is("(2")) {
            if (t.size() > 1) r.dim = (int)std::strtol(t[1].b, nullptr, 10);
            if (r.dim != 3) { err = "only 3-D cases are read"; return false; }
        } else if (s.is("(10")) {
            if (t.size() < 4) continue;
            if (t[1].is("(labels")) continue;
            const long long lo = t[2].hex(), hi = t[3].hex();
            if (t[1].is("(0")) {
                if (hi < 0 || hi > 0x7fffffff / 3) { err = "bad node count"; return false; }
                r.npoint = (int)hi;
                r.P.assign((size_t)hi * 3, 0.0);
                haveNodes = true;
                continue;
            }
            if (!haveNodes || lo < 1 || hi > r.npoint) { err = "node section outside the declared nodes"; return false; }
            long long step = lo - 1;
            while (step < hi && L.next(lb, le)) {
                if (blankOrParen(lb, le, 2)) continue;
                std::string line(lb, le);
                const char* p = line.c_str();
                char* q = nullptr;
                for (int k = 0; k < 3; ++k) {
                    r.P[(size_t)step * 3 + k] = std::strtod(p, &q);
                    if (q == p) { err = "bad node coordinate"; return false; }
                    p = q;
                }
                ++step;
            }
        } else if (s.is("(12")) {
            zoneHeader(t, 12, r);
            if (t.size() < 4 || t[1].is("(labels")) continue;
            const long long lo = t[2].hex(), hi = t[3].hex();
            if (t[1].is("(0")) {
                if (hi < 0 || hi > 0x7fffffff) { err = "bad cell count"; return false; }
                r.ncell = (int)hi;
                r.cellType.assign((size_t)hi, 0);
                haveCells = true;
                continue;
            }
            if (!haveCells || lo < 1) { err = "cell section before the cell declaration"; return false; }
            if (t.size() < 6) continue;
            const Tok& ty = t[5];
            if (ty.is("0)(")) {
                // mixed zone: one element type per cell on the following lines
                long long nx = lo - 1;
                while (nx < hi && L.next(lb, le)) {
                    if (blankOrParen(lb, le, 1)) continue;
                    tokens(lb, le, u);
                    for (const Tok& x : u) {
                        if (nx >= hi) break;
                        char* q = nullptr;
                        const long v = std::strtol(x.b, &q, 10);
                        if (q == x.b) break;
                        if (nx >= 0 && nx < r.ncell) r.cellType[(size_t)nx] = (int)v;
                        ++nx;
                    }
                }
            } else {
                const int v = (int)std::strtol(ty.b, nullptr, 10);
                for (long long i = lo - 1; i < hi && i < r.ncell; ++i) r.cellType[(size_t)i] = v;
            }
        } else if (s.is("(13")) {
            zoneHeader(t, 13, r);
            if (t.size() < 4 || t[1].is("(labels")) continue;
            const long long lo = t[2].hex(), hi = t[3].hex();
            if (t[1].is("(0")) {
                if (hi < 0 || hi > 0x7fffffff) { err = "bad face count"; return false; }
                r.nface = (int)hi;
                r.fnode.assign((size_t)hi * 4, -1);
                r.ftype.assign((size_t)hi, 0);
                r.c0.assign((size_t)hi, -1);
                r.c1.assign((size_t)hi, -1);
                r.ftag.assign((size_t)hi, 0);
                r.fset.assign((size_t)hi, 0);
                haveFaces = true;
                continue;
            }
            if (!haveFaces || lo < 1 || hi > r.nface) { err = "face section outside the declared faces"; return false; }
            if (t.size() < 6) { err = "bad face section header"; return false; }
            const int tag = (int)t[1].hex();
            const int given = (int)std::strtol(t[5].b, nullptr, 10);   // "type)(": 0 mixed, 3 or 4
            long long step = lo - 1;
            while (step < hi && L.next(lb, le)) {
                if (blankOrParen(lb, le, 2)) continue;
                tokens(lb, le, u);
                size_t k = 0;
                int type = given;
                if (given == 0) {
                    if (u.empty()) { err = "bad mixed face line"; return false; }
                    type = (int)std::strtol(u[0].b, nullptr, 10);
                    k = 1;
                }
                if (type != 3 && type != 4) { err = "faces must have 3 or 4 nodes"; return false; }
                if (u.size() < k + (size_t)type + 2) { err = "short face line"; return false; }
                for (int q = 0; q < type; ++q) r.fnode[(size_t)step * 4 + q] = (int)(u[k + q].hex() - 1);
                r.c0[(size_t)step] = (int)(u[k + type].hex() - 1);
                r.c1[(size_t)step] = (int)(u[k + type + 1].hex() - 1);
                r.ftype[(size_t)step] = type;
                r.ftag[(size_t)step] = tag;
                r.fset[(size_t)step] = 1;
                ++step;
            }
        }
    }
    if (!haveNodes || !haveCells || !haveFaces) { err = "the case lacks nodes, cells or faces"; return false; }
    for (int f = 0; f < r.nface; ++f) {
        if (!r.fset[(size_t)f]) { err = "face " + std::to_string(f + 1) + " is declared but not given"; return false; }
        for (int q = 0; q < r.ftype[(size_t)f]; ++q) {
            const int n = r.fnode[(size_t)f * 4 + q];
            if (n < 0 || n >= r.npoint) { err = "face node out of range"; return false; }
        }
        if (r.c0[(size_t)f] < 0 || r.c0[(size_t)f] >= r.ncell || r.c1[(size_t)f] >= r.ncell) {
            err = "face cell out of range";
            return false;
        }
    }
    return true;
}

// ---------------------------------------------------------------------------
// DSMC arrays (setFaceCellNew / preprocess / the DSMC topology)
// ---------------------------------------------------------------------------
bool buildMesh(const Raw& r, DsmcMeshFile& m, std::string& err)
{
    const int nf = r.nface, nc = r.ncell;
    const double* P = r.P.data();
    std::vector<double> cen((size_t)nf * 3), nrm((size_t)nf * 3), area((size_t)nf);
    // face geometry (src/meshImport.cpp:596-668)
    for (int f = 0; f < nf; ++f) {
        const int t = r.ftype[(size_t)f];
        const int* fn = &r.fnode[(size_t)f * 4];
        double c[3] = {0.0, 0.0, 0.0};
        for (int q = 0; q < t; ++q)
            for (int d = 0; d < 3; ++d) c[d] += P[(size_t)fn[q] * 3 + d] / t;
        double cs[3] = {0.0, 0.0, 0.0}, sf[3] = {0.0, 0.0, 0.0}, a = 0.0;
        for (int q = 0; q < t; ++q) {
            const double* X1 = P + (size_t)fn[q] * 3;
            const double* X2 = P + (size_t)fn[q < t - 1 ? q + 1 : 0] * 3;
            double lc[3], l[3], rr[3];
            for (int d = 0; d < 3; ++d) {
                lc[d] = (X1[d] + X2[d] + c[d]) / 3;
                l[d] = X1[d] - c[d];
                rr[d] = X2[d] - c[d];
            }
            double vx = rr[1] * l[2] - rr[2] * l[1];
            double vy = rr[2] * l[0] - l[2] * rr[0];
            double vz = rr[0] * l[1] - l[0] * rr[1];
            vx *= 0.5;
            vy *= 0.5;
            vz *= 0.5;
            const double la = std::sqrt(vx * vx + vy * vy + vz * vz);
            for (int d = 0; d < 3; ++d) cs[d] += la * lc[d];
            sf[0] += vx;
            sf[1] += vy;
            sf[2] += vz;
            a += la;
        }
        for (int d = 0; d < 3; ++d) cen[(size_t)f * 3 + d] = cs[d] / a;
        const double dS = std::sqrt(sf[0] * sf[0] + sf[1] * sf[1] + sf[2] * sf[2]);
        for (int d = 0; d < 3; ++d) nrm[(size_t)f * 3 + d] = sf[d] / dS;
        area[(size_t)f] = a;
    }
    // ghost ids for boundary faces in file order (readFaces)
    std::vector<int> c1(r.c1);
    int bc = 0;
    std::vector<int> bcFaces;
    for (int f = 0; f < nf; ++f)
        if (c1[(size_t)f] < 0) {
            c1[(size_t)f] = nc + bc++;
            bcFaces.push_back(f);
        }
    // cell2face / cell2cell / sgn in face order (src/meshImport.cpp:671-687)
    m.cells.assign((size_t)nc, DsmcCellRec{});
    std::vector<int> tag((size_t)nc, 0);
    for (int c = 0; c < nc; ++c) {
        DsmcCellRec& cr = m.cells[(size_t)c];
        for (int j = 0; j < 6; ++j) { cr.cell2face[j] = -1; cr.cell2cell[j] = -1; cr.cell2face_sgn[j] = -1; }
    }
    auto addFace = [&](int c, int f, int other, int sg) {
        int& k = tag[(size_t)c];
        if (k >= 6) return false;
        DsmcCellRec& cr = m.cells[(size_t)c];
        cr.cell2face[k] = f;
        cr.cell2cell[k] = other;
        cr.cell2face_sgn[k] = sg;
        ++k;
        return true;
    };
    for (int f = 0; f < nf; ++f) {
        const int a0 = r.c0[(size_t)f], a1 = c1[(size_t)f];
        if (a1 < nc && !addFace(a1, f, a0, -1)) { err = "a cell has more than 6 faces"; return false; }
        if (!addFace(a0, f, a1, 1)) { err = "a cell has more than 6 faces"; return false; }
    }
    // volumes and centroids (src/meshImport.cpp:688-723)
    std::vector<double> cellXY((size_t)nc * 3);
    for (int c = 0; c < nc; ++c) {
        DsmcCellRec& cr = m.cells[(size_t)c];
        const int T = tag[(size_t)c];
        if (T == 0) { err = "a cell has no faces"; return false; }
        double cc[3] = {0.0, 0.0, 0.0};
        for (int j = 0; j < T; ++j)
            for (int d = 0; d < 3; ++d) cc[d] += cen[(size_t)cr.cell2face[j] * 3 + d] / T;
        double vcs[3] = {0.0, 0.0, 0.0}, vs = 0.0;
        for (int j = 0; j < T; ++j) {
            const int f = cr.cell2face[j];
            const double* fc = &cen[(size_t)f * 3];
            const double* n = &nrm[(size_t)f * 3];
            const double Cf[3] = {fc[0] - cc[0], fc[1] - cc[1], fc[2] - cc[2]};
            const double lv = std::fabs(n[0] * Cf[0] + n[1] * Cf[1] + n[2] * Cf[2]) * area[(size_t)f] / 3;
            for (int d = 0; d < 3; ++d) vcs[d] += (0.75 * fc[d] + 0.25 * cc[d]) * lv;
            vs += lv;
        }
        cr.num = T;
        cr.fluentCellType = r.cellType[(size_t)c];
        cr.area = vs;
        cr.no = 0;
        for (int d = 0; d < 3; ++d) {
            cellXY[(size_t)c * 3 + d] = vcs[d] / vs;
            cr.cellXY[d] = cellXY[(size_t)c * 3 + d];
        }
    }
    // normals from c0 to c1, ghosts mirrored through their face
    // (preprocess, src/meshImport.cpp:756-783)
    std::vector<double> ghost((size_t)bc * 3);
    for (int k = 0; k < bc; ++k) {
        const int f = bcFaces[(size_t)k];
        const int a0 = r.c0[(size_t)f];
        for (int d = 0; d < 3; ++d) ghost[(size_t)k * 3 + d] = 2 * cen[(size_t)f * 3 + d] - cellXY[(size_t)a0 * 3 + d];
    }
    auto centre = [&](int c) { return c < nc ? &cellXY[(size_t)c * 3] : &ghost[(size_t)(c - nc) * 3]; };
    for (int f = 0; f < nf; ++f) {
        const double* xl = centre(r.c0[(size_t)f]);
        const double* xr = centre(c1[(size_t)f]);
        const double dx = xl[0] - xr[0], dy = xl[1] - xr[1], dz = xl[2] - xr[2];
        const double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
        const double rij[3] = {(xr[0] - xl[0]) / dist, (xr[1] - xl[1]) / dist, (xr[2] - xl[2]) / dist};
        double* n = &nrm[(size_t)f * 3];
        const double vn = n[0] * rij[0] + n[1] * rij[1] + n[2] * rij[2];
        if (vn < 0) { n[0] = -n[0]; n[1] = -n[1]; n[2] = -n[2]; }
    }
    double asum = 0.0;
    for (int c = 0; c < nc; ++c) asum += m.cells[(size_t)c].area;
    // shortest face edge (setParticleMessage)
    double me = DBL_MAX;
    for (int f = 0; f < nf; ++f) {
        const int t = r.ftype[(size_t)f];
        const int* fn = &r.fnode[(size_t)f * 4];
        for (int q = 0; q < t; ++q) {
            const double* a = P + (size_t)fn[q] * 3;
            const double* b = P + (size_t)fn[q < t - 1 ? q + 1 : 0] * 3;
            const double d = std::sqrt((a[0] - b[0]) * (a[0] - b[0]) + (a[1] - b[1]) * (a[1] - b[1]) +
                                       (a[2] - b[2]) * (a[2] - b[2]));
            me = std::min(me, d);
        }
    }
    m.edges.assign((size_t)nf, DsmcEdgeRec{});
    for (int f = 0; f < nf; ++f) {
        DsmcEdgeRec& e = m.edges[(size_t)f];
        e.faceTag = r.ftag[(size_t)f];
        e.faceType = r.ftype[(size_t)f];
        e.length = area[(size_t)f];
        for (int q = 0; q < 4; ++q) e.faceMap[q] = r.fnode[(size_t)f * 4 + q];
        if (e.faceType == 3) e.faceMap[3] = -1;
        e.faceMap[4] = r.c0[(size_t)f];
        e.faceMap[5] = c1[(size_t)f];
        for (int d = 0; d < 3; ++d) {
            e.edgeNormal[d] = nrm[(size_t)f * 3 + d];
            e.edgeCenter[d] = cen[(size_t)f * 3 + d];
        }
    }
    // quad split tags (choose_face_level_quad_split_tag,
    // src/meshImportDsmcTopology.cpp:85-147)
    m.split.assign((size_t)nf, DSMC_FACE_SPLIT_INVALID);
    for (int f = 0; f < nf; ++f) {
        if (r.ftype[(size_t)f] != 4) continue;
        const int* fn = &r.fnode[(size_t)f * 4];
        auto triNormal = [&](int a, int b, int c, double n[3], double& ln) {
            const double* A = P + (size_t)fn[a] * 3;
            const double* B = P + (size_t)fn[b] * 3;
            const double* C = P + (size_t)fn[c] * 3;
            const double e1[3] = {B[0] - A[0], B[1] - A[1], B[2] - A[2]};
            const double e2[3] = {C[0] - A[0], C[1] - A[1], C[2] - A[2]};
            n[0] = e1[1] * e2[2] - e1[2] * e2[1];
            n[1] = e1[2] * e2[0] - e1[0] * e2[2];
            n[2] = e1[0] * e2[1] - e1[1] * e2[0];
            ln = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            return std::isfinite(ln) && ln > 1.0e-30;
        };
        auto score = [&](const int ta[3], const int tb[3]) {
            double n0[3], n1[3], l0, l1;
            const bool ok0 = triNormal(ta[0], ta[1], ta[2], n0, l0);
            const bool ok1 = triNormal(tb[0], tb[1], tb[2], n1, l1);
            if (!(ok0 && ok1)) return DBL_MAX;
            double cosang = (n0[0] * n1[0] + n0[1] * n1[1] + n0[2] * n1[2]) / (l0 * l1);
            cosang = std::min(1.0, std::max(-1.0, cosang));
            return (1.0 - cosang) * 16.0 + std::fabs(l0 - l1) / (l0 + l1);
        };
        static const int a02[3] = {0, 1, 2}, b02[3] = {0, 2, 3}, a13[3] = {0, 1, 3}, b13[3] = {1, 2, 3};
        const double s02 = score(a02, b02), s13 = score(a13, b13);
        const double big = DBL_MAX * 0.5;
        const bool v02 = s02 < big, v13 = s13 < big;
        const bool use13 = !v02 || (v13 && s13 + 1.0e-12 < s02);
        m.split[(size_t)f] = (!v02 && !v13) ? DSMC_FACE_SPLIT_02 : (use13 ? DSMC_FACE_SPLIT_13 : DSMC_FACE_SPLIT_02);
    }
    m.points = r.P;
    m.zones = r.zones;
    m.areaSum = asum;
    m.minEdge = me;
    m.bcnumber = bc;
    return true;
}

// ---------------------------------------------------------------------------
// text output in the reference's ofstream formats
// ---------------------------------------------------------------------------
struct Out {
    FILE* f = nullptr;
    ~Out() { if (f) std::fclose(f); }
    // operator<< of a double at the stream's precision (%g)
    void num(double v, int prec) { std::fprintf(f, "%.*g", prec, v); }
    void str(const char* s) { std::fputs(s, f); }
    void i(long long v) { std::fprintf(f, "%lld", v); }
};

bool findCellZone(const DsmcZone* zones, int32_t nzones, int& id, int& first, int& last)
{
    // out2Fluent_dsmc takes the last zone declaration with id 2
    bool found = false;
    for (int k = 0; k < nzones; ++k)
        if (zones[k].id == 2) {
            id = zones[k].id;
            first = zones[k].first;
            last = zones[k].last;
            found = true;
        }
    return found;
}

int roleOfTag(const DsmcCaseParams* p, int tag)
{
    for (int z = 0; z < p->nzones && z < DSMC_MAX_ZONES; ++z)
        if (p->zone_tag[z] == tag) return p->zone_role[z];
    return DSMC_ROLE_NONE;
}

void normalize3(double v[3])   // ProcessDSMC::normalize, src/ProcessDSMC.cpp:1564-1570
{
    const double len = std::sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= len;
    v[1] /= len;
    v[2] /= len;
}

}  // namespace

extern "C" {

const char* dsmc_meshio_last_error(void) { return g_err.c_str(); }

int dsmc_mesh_read_cas(const char* path, DsmcMeshFile** out)
try {
    if (!out) return failWith("null output");
    *out = nullptr;
    if (!path) return failWith("null path");
    std::unique_ptr<FILE, FileCloser> f(std::fopen(path, "rb"));
    if (!f) return failWith(std::string("cannot open ") + path + ": " + std::strerror(errno));
    std::vector<char> buf;
    char chunk[1 << 16];
    size_t n;
    while ((n = std::fread(chunk, 1, sizeof chunk, f.get())) > 0) buf.insert(buf.end(), chunk, chunk + n);
    f.reset();
    Raw r;
    std::string err;
    if (!parseCas(buf.data(), buf.data() + buf.size(), r, err)) return failWith(std::string(path) + ": " + err);
    std::unique_ptr<DsmcMeshFile> m(new DsmcMeshFile());
    if (!buildMesh(r, *m, err)) return failWith(std::string(path) + ": " + err);
    *out = m.release();
    return DSMC_OK;
}
DSMC_MESHIO_CATCH

void dsmc_mesh_free(DsmcMeshFile* m) { delete m; }

int dsmc_mesh_get_desc(const DsmcMeshFile* m, DsmcMeshDesc* md)
{
    if (!m || !md) return failWith("null argument");
    md->ncell = (int32_t)m->cells.size();
    md->nface = (int32_t)m->edges.size();
    md->npoint = (int32_t)(m->points.size() / 3);
    md->cells = m->cells.data();
    md->edges = m->edges.data();
    md->localPointXY = m->points.data();
    md->faceSplitTag = m->split.data();
    return DSMC_OK;
}

int dsmc_mesh_get_zones(const DsmcMeshFile* m, DsmcZone* zones, int32_t capacity, int32_t* count)
{
    if (!m || !count) return failWith("null argument");
    *count = (int32_t)m->zones.size();
    if (zones)
        for (int32_t k = 0; k < capacity && k < *count; ++k) zones[k] = m->zones[(size_t)k];
    return DSMC_OK;
}

int dsmc_mesh_get_stats(const DsmcMeshFile* m, double* area_sum, double* min_edge, int32_t* bcnumber)
{
    if (!m) return failWith("null argument");
    if (area_sum) *area_sum = m->areaSum;
    if (min_edge) *min_edge = m->minEdge;
    if (bcnumber) *bcnumber = m->bcnumber;
    return DSMC_OK;
}

int dsmc_mesh_message(const DsmcMeshFile* m, double Ma, double Kn, int32_t ppc, double L0, double T_in, double T_wall,
                      double cfl, double cfl_ns, DsmcMeshMessage* out)
try {
    if (!m || !out) return failWith("null argument");
    if (!(Kn > 0.0) || !(L0 > 0.0) || !(T_in > 0.0) || ppc <= 0) return failWith("Kn, L0, T_in and ppc must be positive");
    DsmcMeshMessage g{};
    const double pi = M_PI;
    const int ncell = (int)m->cells.size(), nface = (int)m->edges.size();
    // setMa_Kn_CFL and the gas model of setMeshMessage (src/meshImport.cpp:1252-1330)
    const double dr = 2.0, dv = 1.626, zr = 3.5, zv = 2 * zr, omega = 0.74;
    const double f_tra = 2.365, f_rot = 1.435;
    const double gamma = (5.0 + dr) / (3.0 + dr);
    const double delta_sm = 1.0 / 1.33;
    g.Ncell = ncell;
    g.Nface = nface;
    g.Npoint = (int32_t)(m->points.size() / 3);
    g.Nk = 0;
    g.bcnumber = m->bcnumber;
    g.Nghost = ncell + m->bcnumber;
    g.Ma = Ma;
    g.Kn = Kn;
    g.cfl = cfl;
    g.Area = m->areaSum;
    g.gamma = gamma;
    g.omega = omega;
    g.dr = dr;
    g.dv = dv;
    g.zr = zr;
    g.zv = zv;
    g.var = 6;
    g.qn = 2;
    g.cfl_ns = cfl_ns;
    g.f_tra = f_tra;
    g.f_rot = f_rot;
    g.pr = (5.0 + dr) * 0.5 / (1.5 * f_tra + dr * 0.5 * f_rot);
    g.delta_rp = std::pow(pi * 0.5, 0.5) / Kn;
    g.delta_sm = delta_sm;
    g.omeag0 = 1.0 - 2.0 * zr * (2.5 / f_tra - 1.0);
    g.omeag1 = 1 - (1 / (f_rot * delta_sm) - 1) * (delta_sm / (1 - delta_sm)) * zr;
    g.cv = 1 / (gamma - 1.0);
    g.cp = g.cv * gamma;
    g.eNface = m->bcnumber;
    g.iNface = nface - m->bcnumber;
    // reference state (src/meshImport.cpp:1316-1360)
    const double kB = 1.3806e-23, T_ref = 273.15, p_mass = 4.65e-26;
    const double d_ref = 4.17e-10, alpha = 1.0;
    const double v_rms = std::sqrt(2 * kB * T_ref / p_mass);
    const double v_in = std::sqrt(2 * kB * T_in / p_mass);
    const double d_ref2 = d_ref * d_ref;
    double miu_ref = 5.0 * (alpha + 1.0) * (alpha + 2.0) * std::sqrt(p_mass * kB * T_ref / pi) / 4.0 / alpha /
                     (5.0 - 2.0 * omega) / (7.0 - 2.0 * omega) / d_ref2;
    miu_ref *= std::pow(T_in / T_ref, omega);
    const double p_ref = miu_ref / (Kn * L0) * std::sqrt(pi * kB / p_mass * T_in / 2.0);
    const double n_ref = p_ref / (kB * T_in);
    const double dt_ref = (1 / Kn) * std::sqrt(pi) / 2 * miu_ref / p_ref * std::sqrt(T_in / T_ref);
    g.kB = kB;
    g.T_ref = T_ref;
    g.T_in = T_in;
    g.v_in = v_in;
    g.n_ref = n_ref;
    g.p_ref = p_ref;
    g.d_ref = d_ref;
    g.p_mass = p_mass;
    g.p_mass_r = 0.5 * p_mass;
    g.miu_ref = miu_ref;
    g.v_rms = v_rms;
    g.eta = omega - 0.5;
    g.Twall_ref = T_wall / T_ref;
    g.alpha = alpha;
    g.P_relax = 0.18;
    g.dt_ref = dt_ref;
    // setParticleMessage (src/meshImport.cpp:1365-1405)
    const double nps = (double)((long long)ppc * (long long)ncell);
    g.Neff = m->areaSum * n_ref / nps;
    g.dtime = m->minEdge * 0.2;
    *out = g;
    return DSMC_OK;
}
DSMC_MESHIO_CATCH

int dsmc_write_fluent_cells(const char* path, const DsmcMeshMessage* mess, const DsmcZone* zones, int32_t nzones,
                            const double* w, int32_t ncell)
try {
    if (!path || !mess || !zones || !w) return failWith("null argument");
    int id = 0, first = 0, last = 0;
    if (!findCellZone(zones, nzones, id, first, last)) return failWith("no cell zone with id 2");
    if (first < 1 || last > ncell || first > last + 1) return failWith("cell zone range outside the fields");
    double ts = mess->T_in / mess->T_ref;
    if (!(ts > 0.0) || !std::isfinite(ts)) ts = 1.0;
    double vs = std::sqrt(mess->gamma / 2.0) * mess->v_in / mess->v_rms;
    if (!(vs > 0.0) || !std::isfinite(vs)) vs = 1.0;
    const double ss = ts, hs = ts * vs;
    Out o;
    o.f = std::fopen(path, "w");
    if (!o.f) return failWith(std::string("cannot write ") + path + ": " + std::strerror(errno));
    o.str("(0 \" (300 (var-id zone-id var-size 0 0 first-id last-id)(......))\" )\n");
    auto head = [&](int var, int size) {
        std::fprintf(o.f, "(300 (%d %d %d 0 0 %d %d)\n(\n", var, id, size, first, last);
    };
    // 700: density
    head(700, 1);
    for (int c = first - 1; c < last; ++c) { o.num(w[(size_t)c * 18 + 0], 6); o.str("\n"); }
    o.str("))\n");
    // 701: velocity (trailing blank kept)
    head(701, 3);
    for (int c = first - 1; c < last; ++c) {
        for (int k = 1; k <= 3; ++k) { o.num(w[(size_t)c * 18 + k] / vs, 6); o.str(" "); }
        o.str("\n");
    }
    o.str("))\n");
    // 702: T, Tr
    head(702, 2);
    for (int c = first - 1; c < last; ++c) {
        o.num(w[(size_t)c * 18 + 4] / ts, 6); o.str(" ");
        o.num(w[(size_t)c * 18 + 14] / ts, 6); o.str(" \n");
    }
    o.str("))\n");
    // 710: stress
    head(710, 6);
    for (int c = first - 1; c < last; ++c) {
        for (int k = 5; k <= 10; ++k) { o.num(w[(size_t)c * 18 + k] / ss, 6); o.str(" "); }
        o.str("\n");
    }
    o.str("))\n");
    // 711, 712: heat fluxes
    for (int var : {711, 712}) {
        const int k0 = var == 711 ? 11 : 15;
        head(var, 3);
        for (int c = first - 1; c < last; ++c) {
            o.num(w[(size_t)c * 18 + k0] / hs, 6); o.str(" ");
            o.num(w[(size_t)c * 18 + k0 + 1] / hs, 6); o.str(" ");
            o.num(w[(size_t)c * 18 + k0 + 2] / hs, 6); o.str("\n");
        }
        o.str("))\n");
    }
    if (std::ferror(o.f)) return failWith(std::string("write error on ") + path);
    return DSMC_OK;
}
DSMC_MESHIO_CATCH

int dsmc_write_fluent_wall(const char* path, const DsmcMeshMessage* mess, const DsmcCaseParams* params,
                           const DsmcZone* zones, int32_t nzones, const DsmcEdgeRec* edges, int32_t nface,
                           const double* tally, int32_t istep)
try {
    if (!path || !mess || !params || !edges || !tally || (nzones > 0 && !zones)) return failWith("null argument");
    if (nface <= 0) return failWith("no faces");
    const bool steady = istep > params->nss;
    const double sampleSteps = steady ? (double)(istep - params->nss) : 1.0;
    const double timeScale = (mess->dtime > 0.0 && sampleSteps > 0.0) ? mess->Neff / (mess->dtime * sampleSteps) : 0.0;
    struct F { double stress[3], normal[3], pressure, shear[3], qt, qr, q; };
    std::vector<F> out((size_t)nface, F{});
    std::vector<char> wall((size_t)nface, 0);
    for (int f = 0; f < nface; ++f) {
        const DsmcEdgeRec& e = edges[f];
        if (roleOfTag(params, e.faceTag) != DSMC_ROLE_WALL) continue;
        wall[(size_t)f] = 1;
        double no[3] = {e.edgeNormal[0], e.edgeNormal[1], e.edgeNormal[2]};
        const double len = std::sqrt(no[0] * no[0] + no[1] * no[1] + no[2] * no[2]);
        if (len > 0.0 && std::isfinite(len)) normalize3(no);
        else { no[0] = 1.0; no[1] = 0.0; no[2] = 0.0; }
        double ni[3] = {-no[0], -no[1], -no[2]};
        normalize3(ni);
        const double* in = tally + (size_t)f * 6;
        const double pn = in[1] * ni[0] + in[2] * ni[1] + in[3] * ni[2];
        const double pt[3] = {in[1] - pn * ni[0], in[2] - pn * ni[1], in[3] - pn * ni[2]};
        const double area = (e.length > 0.0 && std::isfinite(e.length)) ? e.length : 1.0;
        const double scale = (area > 0.0 && mess->n_ref > 0.0) ? 2.0 * timeScale / area / mess->n_ref : 0.0;
        F& o = out[(size_t)f];
        for (int d = 0; d < 3; ++d) o.normal[d] = no[d];
        o.pressure = pn * scale;
        for (int d = 0; d < 3; ++d) o.shear[d] = -pt[d] * scale;
        for (int d = 0; d < 3; ++d) o.stress[d] = o.pressure * o.normal[d] + o.shear[d];
        o.qt = -in[4] * scale;
        o.qr = -in[5] * scale;
        o.q = o.qt + o.qr;
    }
    struct Block { int id, first, last; };
    std::vector<Block> blocks;
    for (int k = 0; k < nzones; ++k) {
        const int first = std::max(1, (int)zones[k].first);
        const int last = std::min((int)zones[k].last, (int)nface);
        if (first > last) continue;
        bool all = true;
        for (int f = first - 1; f < last && all; ++f) all = wall[(size_t)f] != 0;
        if (all) blocks.push_back(Block{zones[k].id, first, last});
    }
    if (blocks.empty()) return DSMC_OK;
    Out o;
    o.f = std::fopen(path, "w");
    if (!o.f) return failWith(std::string("cannot write ") + path + ": " + std::strerror(errno));
    o.str("(0 \" (300 (var-id zone-id var-size 0 0 first-id last-id)(......))\" )\n");
    o.str("(0 \"DSMC normalized wall fields: 700 stress vector, 701 q_trans, 702 q_rot, 703 normal vector, 704 "
          "pressure, 705 shear vector, 706 q_total\")\n");
    for (const Block& b : blocks) {
        auto vec = [&](int var, double (F::*field)[3]) {
            std::fprintf(o.f, "(300 (%d %d 3 0 0 %d %d)\n(\n", var, b.id, b.first, b.last);
            for (int f = b.first - 1; f < b.last; ++f) {
                const double* v = out[(size_t)f].*field;
                o.num(v[0], 16); o.str(" "); o.num(v[1], 16); o.str(" "); o.num(v[2], 16); o.str("\n");
            }
            o.str("))\n");
        };
        auto sca = [&](int var, double F::*field) {
            std::fprintf(o.f, "(300 (%d %d 1 0 0 %d %d)\n(\n", var, b.id, b.first, b.last);
            for (int f = b.first - 1; f < b.last; ++f) { o.num(out[(size_t)f].*field, 16); o.str("\n"); }
            o.str("))\n");
        };
        vec(700, &F::stress);
        sca(701, &F::qt);
        sca(702, &F::qr);
        vec(703, &F::normal);
        sca(704, &F::pressure);
        vec(705, &F::shear);
        sca(706, &F::q);
    }
    if (std::ferror(o.f)) return failWith(std::string("write error on ") + path);
    return DSMC_OK;
}
DSMC_MESHIO_CATCH

}  // extern "C"
