/*
 * dsmc_oracle.c — CPU restatement of the reference's DSMC particle step.
 * ORACLE TEST INFRASTRUCTURE (see dsmc_oracle.h); never part of the product.
 *
 * Citations are to the reference's src/ files.
 */
#include "dsmc_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

/* byte layouts of the reference's records (src/meshImport.h:168-208) */
typedef struct {
    int32_t num, fluentCellType;
    int32_t cell2face[6], cell2cell[6], cell2face_sgn[6];
    double area;
    int32_t no;
    double cellXY[3];
} Cell;
typedef struct {
    int32_t faceTag, faceType;
    double length;
    int32_t faceMap[6];
    double edgeNormal[3], edgeCenter[3];
} Edge;
typedef struct {
    int32_t Ncell, Nface, Npoint, Nk, bcnumber, Nghost;
    double Area, Ma, Kn, cfl, gamma, dr, dv, zr, zv, omega;
    int32_t var, qn;
    double f_tra, f_rot, delta_rp, delta_sm, omeag0, omeag1, cfl_ns, pr, cp, cv;
    double kB, p_mass, p_mass_r, T_ref, n_ref, miu_ref, Twall_ref, p_ref, d_ref;
    double alpha, v_rms, eta, P_relax, dt_ref, T_in, v_in;
    int32_t eNface, iNface;
    double Neff, dtime;
} Mess;

enum { R_NONE = 0, R_INTERFACE, R_INLET, R_OUTLET, R_WALL, R_SPECULAR };
enum { T_STAY = 0, T_MOVED = 1, T_REMOVED = -1, T_DROPPED = -2, T_LOST = -3 };
enum { K_INJ = 0, K_REM, K_DROP, K_LOST, K_WALL, K_CROSS, K_PAIRS, K_COLL };

typedef struct {
    int cell, edge, tag;
    double geom[9], rot[9], gas[8], addBase;
} Patch;

struct OracleCase {
    int ncell, nface, npoint;
    Cell* cells;
    Edge* edges;
    double* pts;
    unsigned char* split;
    Mess m;
    int* role;
    int* faceWall;
    double* wallRot;      /* [nwall][2][9] */
    int nwall;
    int* triOff;          /* [ncell+1] */
    double* tri;          /* [ntri][9] */
    int* triFace;
    int* triTag;
    int ntri;
    signed char* rev;     /* [ncell][6] */
    Patch* patches;
    int npatch;
    double dirx, diry;
    int nss, nscheme, nevery, nrepeat, wallStats, maxCross;
    uint32_t k0, k1;
    double cdPrefactor;
    /* particles, canonical order */
    int64_t n, cap;
    double *px, *py, *pz, *vx, *vy, *vz, *ir;
    int* pc;
    int* start;           /* [ncell+1] */
    /* after inject / move, before the sort */
    int64_t nInj;
    int sorted;
    /* per-cell state */
    double *crmax, *remColl, *remInj, *acc, *record, *local, *finalRecord, *stepMom, *wsamp, *wall;
    char* wvalid;
    unsigned char* sparse;
    int* saccum;
    int localLazy, lastIstep;
    uint64_t ctr[8];
    uint32_t gsisEpoch;   /* GSIS updates made so far (keys their random streams) */
};

/* ------------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon et al., SC'11)                                      */
/* ------------------------------------------------------------------------ */
void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c0 = ctr[0], c1 = ctr[1], c2 = ctr[2], c3 = ctr[3];
    uint32_t k0 = key[0], k1 = key[1];
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c0;
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c2;
        const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        const uint32_t n0 = hi1 ^ c1 ^ k0, n1 = lo1, n2 = hi0 ^ c3 ^ k1, n3 = lo0;
        c0 = n0; c1 = n1; c2 = n2; c3 = n3;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

typedef struct {
    uint32_t id, step, purpose, n, k0, k1;
    uint32_t buf[4];
    int avail;
} Stream;

static void st_init(Stream* s, uint32_t id, uint32_t step, uint32_t purpose, uint32_t k0, uint32_t k1)
{
    s->id = id; s->step = step; s->purpose = purpose; s->n = 0; s->k0 = k0; s->k1 = k1; s->avail = 0;
}
static uint32_t st_next(Stream* s)
{
    if (s->avail == 0) {
        const uint32_t c[4] = {s->id, s->step, s->purpose, s->n};
        const uint32_t k[2] = {s->k0, s->k1};
        oracle_philox(c, k, s->buf);
        s->n++;
        s->avail = 4;
    }
    return s->buf[4 - s->avail--];
}
static double st_u64(Stream* s)
{
    const uint64_t a = st_next(s), b = st_next(s);
    const uint64_t k = (a << 21) ^ (b >> 11);
    return ((double)k + 0.5) * 0x1.0p-53;
}
static uint32_t mulhi(uint32_t a, uint32_t b) { return (uint32_t)(((uint64_t)a * b) >> 32); }

/* ------------------------------------------------------------------------ */
/* geometry helpers                                                          */
/* ------------------------------------------------------------------------ */
static void decode_split(unsigned char tag, int t0[3], int t1[3])   /* src/meshImport.h:309-327 */
{
    if (tag == 0) { t0[0] = 0; t0[1] = 1; t0[2] = 2; t1[0] = 0; t1[1] = 2; t1[2] = 3; }
    else if (tag == 1) { t0[0] = 0; t0[1] = 1; t0[2] = 3; t1[0] = 1; t1[1] = 2; t1[2] = 3; }
    else { t0[0] = t0[1] = t0[2] = -1; t1[0] = t1[1] = t1[2] = -1; }
}
static void normalize3(double v[3])   /* src/ProcessDSMC.cpp:1564-1570 */
{
    const double len = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    v[0] /= len; v[1] /= len; v[2] /= len;
}
static void cross3(const double* a, const double* b, double* r)   /* src/MeshparticalInitial.cpp:819-823 */
{
    r[0] = a[1] * b[2] - a[2] * b[1];
    r[1] = a[2] * b[0] - a[0] * b[2];
    r[2] = a[0] * b[1] - a[1] * b[0];
}
static double dot3(const double* a, const double* b)   /* src/MeshparticalInitial.cpp:829-835 */
{
    double r = 0.0;
    for (int i = 0; i < 3; ++i) r += a[i] * b[i];
    return r;
}
static void rotation(const double* n, double R[9])   /* buildRotationMatrix, src/ProcessDSMC.cpp:1583-1603 */
{
    double t1[3], t2[3];
    if ((fabs(n[0]) <= fabs(n[1])) && (fabs(n[0]) <= fabs(n[2]))) { t1[0] = 0.0; t1[1] = n[2]; t1[2] = -n[1]; }
    else if (fabs(n[1]) < fabs(n[2])) { t1[0] = n[2]; t1[1] = 0.0; t1[2] = -n[0]; }
    else { t1[0] = n[1]; t1[1] = -n[0]; t1[2] = 0.0; }
    normalize3(t1);
    cross3(n, t1, t2);
    normalize3(t2);
    R[0] = t1[0]; R[1] = t2[0]; R[2] = n[0];
    R[3] = t1[1]; R[4] = t2[1]; R[5] = n[1];
    R[6] = t1[2]; R[7] = t2[2]; R[8] = n[2];
}
static int load_point(const OracleCase* o, int idx, double P[3])
{
    if (idx < 0 || idx >= o->npoint) return 0;
    P[0] = o->pts[3 * idx]; P[1] = o->pts[3 * idx + 1]; P[2] = o->pts[3 * idx + 2];
    return 1;
}
/* wallMap normals of a quad face, processFacesQuadNormals, src/ProcessDSMC.cpp:1054-1127 */
static int quad_normals(const OracleCase* o, int f, double n1[3], double n2[3])
{
    const Edge* e = &o->edges[f];
    double P[4][3];
    for (int k = 0; k < 4; ++k)
        if (!load_point(o, e->faceMap[k], P[k])) return 0;
    int t[2][3];
    decode_split(o->split[f], t[0], t[1]);
    if (t[0][0] < 0 || t[1][0] < 0) decode_split(0, t[0], t[1]);
    double* outs[2] = {n1, n2};
    for (int s = 0; s < 2; ++s) {
        const double* X = P[t[s][0]];
        const double* Y = P[t[s][1]];
        const double* Z = P[t[s][2]];
        const double a[3] = {Y[0] - X[0], Y[1] - X[1], Y[2] - X[2]};
        const double b[3] = {Z[0] - X[0], Z[1] - X[1], Z[2] - X[2]};
        cross3(a, b, outs[s]);
        normalize3(outs[s]);
        if (dot3(e->edgeNormal, outs[s]) < 0.0) {
            outs[s][0] *= -1.0; outs[s][1] *= -1.0; outs[s][2] *= -1.0;
        }
    }
    return 1;
}

static int role_of(int nz, const int* tag, const int* role, const int* inj, int t, int* inject)
{
    for (int z = 0; z < nz; ++z)
        if (tag[z] == t) { if (inject) *inject = inj[z]; return role[z]; }
    if (inject) *inject = 0;
    return R_NONE;
}

static int cmp_patch(const void* a, const void* b)
{
    const Patch* x = (const Patch*)a;
    const Patch* y = (const Patch*)b;
    if (x->cell != y->cell) return x->cell < y->cell ? -1 : 1;
    /* stable by original order: edge then tag */
    if (x->edge != y->edge) return x->edge < y->edge ? -1 : 1;
    return x->tag < y->tag ? -1 : (x->tag > y->tag);
}

OracleCase* oracle_create(int ncell, int nface, int npoint, const void* cells, const void* edges, const double* points,
                          const unsigned char* split, const void* mess, int nzones, const int* zone_tag,
                          const int* zone_role, const int* zone_inject, double dirx, double diry, int nss, int nscheme,
                          int nevery, int nrepeat, int wall_stats, uint64_t seed, int max_cross)
{
    OracleCase* o = (OracleCase*)calloc(1, sizeof(OracleCase));
    if (!o) return NULL;
    o->ncell = ncell; o->nface = nface; o->npoint = npoint;
    o->cells = (Cell*)malloc(sizeof(Cell) * ncell);
    o->edges = (Edge*)malloc(sizeof(Edge) * nface);
    o->pts = (double*)malloc(sizeof(double) * 3 * npoint);
    o->split = (unsigned char*)malloc(nface);
    memcpy(o->cells, cells, sizeof(Cell) * ncell);
    memcpy(o->edges, edges, sizeof(Edge) * nface);
    memcpy(o->pts, points, sizeof(double) * 3 * npoint);
    if (split) memcpy(o->split, split, nface); else memset(o->split, 255, nface);
    memcpy(&o->m, mess, sizeof(Mess));
    o->dirx = dirx; o->diry = diry;
    o->nss = nss; o->nscheme = nscheme; o->nevery = nevery; o->nrepeat = nrepeat;
    o->wallStats = wall_stats; o->maxCross = max_cross > 0 ? max_cross : 4096;
    o->k0 = (uint32_t)(seed & 0xffffffffu); o->k1 = (uint32_t)(seed >> 32);
    {
        const double conDen = tgamma(5.0 / 2.0 - o->m.omega);   /* src/ProcessDSMC.cpp:2626-2630 */
        const double d2 = o->m.d_ref * o->m.d_ref;
        o->cdPrefactor = M_PI * d2 * pow(2 * o->m.kB * o->m.T_ref / o->m.p_mass_r, o->m.eta) / conDen;
    }
    /* roles and wall slots */
    o->role = (int*)malloc(sizeof(int) * nface);
    o->faceWall = (int*)malloc(sizeof(int) * nface);
    o->wallRot = (double*)malloc(sizeof(double) * 18 * (nface + 1));
    for (int f = 0; f < nface; ++f) {
        o->role[f] = role_of(nzones, zone_tag, zone_role, zone_inject, o->edges[f].faceTag, NULL);
        o->faceWall[f] = -1;
        if (o->role[f] == R_WALL || o->role[f] == R_SPECULAR) {
            /* getWallNormal, src/ProcessDSMC.cpp:1708-1731 */
            double nb[3] = {o->edges[f].edgeNormal[0], o->edges[f].edgeNormal[1], o->edges[f].edgeNormal[2]};
            normalize3(nb);
            double n1[3] = {nb[0], nb[1], nb[2]}, n2[3] = {nb[0], nb[1], nb[2]};
            if (o->edges[f].faceType == 4) {
                double q1[3], q2[3];
                if (quad_normals(o, f, q1, q2)) { memcpy(n1, q1, sizeof n1); memcpy(n2, q2, sizeof n2); }
            }
            const int w = o->nwall++;
            o->faceWall[f] = w;
            rotation(n1, &o->wallRot[(size_t)w * 18]);
            rotation(n2, &o->wallRot[(size_t)w * 18 + 9]);
        }
    }
    /* triangle cache: rebuildFaceTraversalCache, src/ProcessDSMCGeometry.cpp:145-214 */
    o->triOff = (int*)malloc(sizeof(int) * (ncell + 1));
    o->tri = (double*)malloc(sizeof(double) * 9 * 12 * (size_t)ncell);
    o->triFace = (int*)malloc(sizeof(int) * 12 * (size_t)ncell);
    o->triTag = (int*)malloc(sizeof(int) * 12 * (size_t)ncell);
    int nt = 0;
    for (int c = 0; c < ncell; ++c) {
        o->triOff[c] = nt;
        for (int m = 0; m < o->cells[c].num && m < 6; ++m) {
            const int f = o->cells[c].cell2face[m];
            if (f < 0 || f >= nface) continue;
            const Edge* e = &o->edges[f];
            int ids[2][3], tags[2], k = 0;
            if (e->faceType == 3) {
                ids[0][0] = e->faceMap[0]; ids[0][1] = e->faceMap[1]; ids[0][2] = e->faceMap[2]; tags[0] = -1; k = 1;
            } else if (e->faceType == 4) {
                int t0[3], t1[3];
                decode_split(o->split[f], t0, t1);
                if (t0[0] < 0 || t1[0] < 0) decode_split(0, t0, t1);
                for (int q = 0; q < 3; ++q) { ids[0][q] = e->faceMap[t0[q]]; ids[1][q] = e->faceMap[t1[q]]; }
                tags[0] = 1; tags[1] = 2; k = 2;
            }
            for (int s = 0; s < k; ++s) {
                double A[3], B[3], Cc[3];
                if (!load_point(o, ids[s][0], A) || !load_point(o, ids[s][1], B) || !load_point(o, ids[s][2], Cc)) continue;
                double* T = &o->tri[(size_t)nt * 9];
                T[0] = A[0]; T[1] = A[1]; T[2] = A[2];
                T[3] = B[0] - A[0]; T[4] = B[1] - A[1]; T[5] = B[2] - A[2];
                T[6] = Cc[0] - A[0]; T[7] = Cc[1] - A[1]; T[8] = Cc[2] - A[2];
                o->triFace[nt] = f;
                o->triTag[nt] = tags[s];
                ++nt;
            }
        }
    }
    o->triOff[ncell] = nt;
    o->ntri = nt;
    /* reverse neighbour slots */
    o->rev = (signed char*)malloc(6 * (size_t)ncell);
    memset(o->rev, -1, 6 * (size_t)ncell);
    for (int c = 0; c < ncell; ++c)
        for (int j = 0; j < 6 && j < o->cells[c].num; ++j) {
            const int nb = o->cells[c].cell2cell[j];
            const int f = o->cells[c].cell2face[j];
            if (nb < 0 || nb >= ncell) continue;
            for (int p = 0; p < 6 && p < o->cells[nb].num; ++p)
                if (o->cells[nb].cell2face[p] == f) { o->rev[(size_t)c * 6 + j] = (signed char)p; break; }
        }
    /* inlet patches: rebuildBoundaryEmitCache, src/ProcessDSMC.cpp:583-768 */
    o->patches = (Patch*)malloc(sizeof(Patch) * (2 * (size_t)nface + 1));
    o->npatch = 0;
    for (int f = 0; f < nface; ++f) {
        int inject = 0;
        const int r = role_of(nzones, zone_tag, zone_role, zone_inject, o->edges[f].faceTag, &inject);
        if (r != R_INLET || !inject) continue;
        const Edge* e = &o->edges[f];
        int cl = -1;
        if (e->faceMap[4] >= 0 && e->faceMap[4] < ncell) cl = e->faceMap[4];
        if (cl < 0 && e->faceMap[5] >= 0 && e->faceMap[5] < ncell) cl = e->faceMap[5];
        if (cl < 0 || (e->faceType != 3 && e->faceType != 4)) continue;
        const int nn = e->faceType == 4 ? 4 : 3;
        double P[4][3];
        int ok = 1;
        for (int k = 0; k < nn && ok; ++k) ok = load_point(o, e->faceMap[k], P[k]);
        if (!ok) continue;
        int tri[2][3] = {{0, 1, 2}, {-1, -1, -1}};
        int ntris = 1;
        double qn[2][3] = {{0}};
        if (e->faceType == 4) {
            decode_split(o->split[f], tri[0], tri[1]);
            if (tri[0][0] < 0 || tri[1][0] < 0) decode_split(0, tri[0], tri[1]);
            ntris = 2;
            quad_normals(o, f, qn[0], qn[1]);
        }
        for (int tt = 1; tt <= ntris; ++tt) {
            const int s = e->faceType == 4 ? tt - 1 : 0;
            double nrm[3];
            if (e->faceType == 4) { nrm[0] = qn[s][0]; nrm[1] = qn[s][1]; nrm[2] = qn[s][2]; }
            else {
                nrm[0] = e->edgeNormal[0]; nrm[1] = e->edgeNormal[1]; nrm[2] = e->edgeNormal[2];
                const double len = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
                if (len > 0.0 && isfinite(len)) { nrm[0] /= len; nrm[1] /= len; nrm[2] /= len; }
            }
            const double* P0 = P[tri[s][0]];
            const double* P1 = P[tri[s][1]];
            const double* P2 = P[tri[s][2]];
            Patch pt;
            memset(&pt, 0, sizeof pt);
            pt.cell = cl; pt.edge = f; pt.tag = e->faceType == 3 ? -1 : tt;
            for (int d = 0; d < 3; ++d) { pt.geom[d] = P0[d]; pt.geom[3 + d] = P1[d] - P0[d]; pt.geom[6 + d] = P2[d] - P0[d]; }
            const double ax = P1[0] - P0[0], ay = P1[1] - P0[1], az = P1[2] - P0[2];
            const double bx = P2[0] - P0[0], by = P2[1] - P0[1], bz = P2[2] - P0[2];
            const double cx = ay * bz - az * by, cy = az * bx - ax * bz, cz = ax * by - ay * bx;
            const double area = 0.5 * sqrt(cx * cx + cy * cy + cz * cz);
            const double nmag = sqrt(nrm[0] * nrm[0] + nrm[1] * nrm[1] + nrm[2] * nrm[2]);
            if (!(area > 0.0) || !isfinite(area) || !(nmag > 0.0) || !isfinite(nmag)) continue;
            const double neg[3] = {-nrm[0], -nrm[1], -nrm[2]};
            rotation(neg, pt.rot);
            const double* R = pt.rot;
            /* computeBoundaryGasState, src/ProcessDSMC.cpp:2318-2367 */
            const double base = 1.0 * o->m.Ma * sqrt(o->m.gamma / 2.0) * o->m.v_in / o->m.v_rms;
            const double uxN = base * dirx, uyN = base * diry, uzN = 0.0;
            const double tN = o->m.T_in / o->m.T_ref;
            const double rhoP = 1.0 * o->m.n_ref;
            const double uxP = uxN * o->m.v_rms, uyP = uyN * o->m.v_rms, uzP = uzN * o->m.v_rms;
            const double tP = tN * o->m.T_ref;
            const double beta = 1.0 / sqrt(2 * o->m.kB / o->m.p_mass * tP);
            const double sx = uxP * beta, sy = uyP * beta, sz = uzP * beta;
            const double stp1 = R[0] * sx + R[3] * sy + R[6] * sz;
            const double stp2 = R[1] * sx + R[4] * sy + R[7] * sz;
            const double snp = R[2] * sx + R[5] * sy + R[8] * sz;
            const double fs1 = snp + sqrt(snp * snp + 2.0);
            const double fs2 = 0.5 * (1.0 + snp * (2.0 * snp - fs1));
            double QA = 3.0;
            if (fabs(snp) > 3.0) QA = fabs(snp) + 1.0;
            pt.gas[0] = snp; pt.gas[1] = fs1; pt.gas[2] = fs2; pt.gas[3] = stp1; pt.gas[4] = stp2;
            pt.gas[5] = tN; pt.gas[6] = sqrt(tN); pt.gas[7] = QA;
            /* computeBoundaryInsertCount, src/ProcessDSMC.cpp:2380-2403 */
            double cosT = 0.0;
            const double Umag = sqrt(uxP * uxP + uyP * uyP + uzP * uzP);
            if (Umag > 0.0 && nmag > 0.0) cosT = -((uxP * nrm[0] + uyP * nrm[1] + uzP * nrm[2]) / (Umag * nmag));
            const double s_ = beta * Umag;
            const double scos = s_ * cosT;
            const double addNum = o->m.dtime * area * rhoP / 2.0 / sqrt(M_PI) * sqrt(tP / o->m.T_ref) *
                                  (exp(-(scos * scos)) + sqrt(M_PI) * scos * (1.0 + erf(scos)));
            pt.addBase = addNum / o->m.Neff;
            o->patches[o->npatch++] = pt;
        }
    }
    qsort(o->patches, (size_t)o->npatch, sizeof(Patch), cmp_patch);
    /* per-cell state, Collision_constant_initial, src/MeshparticalInitial.cpp:798-810 */
    const size_t nc = (size_t)ncell;
    o->crmax = (double*)malloc(sizeof(double) * nc);
    for (size_t c = 0; c < nc; ++c) o->crmax[c] = 3.0;
    o->remColl = (double*)calloc(nc, sizeof(double));
    o->remInj = (double*)calloc(nc, sizeof(double));
    o->acc = (double*)calloc(nc * 54, sizeof(double));
    o->record = (double*)calloc(nc * 18, sizeof(double));
    o->local = (double*)calloc(nc * 18, sizeof(double));
    o->finalRecord = (double*)calloc(nc * 18, sizeof(double));
    o->stepMom = (double*)calloc(nc * 18, sizeof(double));
    o->wsamp = (double*)calloc(nc, sizeof(double));
    o->wvalid = (char*)calloc(nc, 1);
    o->sparse = (unsigned char*)calloc(nc, 1);
    o->saccum = (int*)calloc(nc, sizeof(int));
    o->wall = (double*)calloc((size_t)(o->nwall + 1) * 6, sizeof(double));
    o->start = (int*)calloc(nc + 1, sizeof(int));
    o->sorted = 1;
    return o;
}

void oracle_destroy(OracleCase* o)
{
    if (!o) return;
    void* ps[] = {o->cells, o->edges, o->pts, o->split, o->role, o->faceWall, o->wallRot, o->triOff, o->tri,
                  o->triFace, o->triTag, o->rev, o->patches, o->px, o->py, o->pz, o->vx, o->vy, o->vz, o->ir,
                  o->pc, o->start, o->crmax, o->remColl, o->remInj, o->acc, o->record, o->local, o->finalRecord,
                  o->stepMom, o->wsamp, o->wall, o->wvalid, o->sparse, o->saccum};
    for (size_t i = 0; i < sizeof ps / sizeof ps[0]; ++i) free(ps[i]);
    free(o);
}

/* ------------------------------------------------------------------------ */
/* tracing                                                                   */
/* ------------------------------------------------------------------------ */
/* intersectCachedTri, src/ProcessDSMC.cpp:1174-1197 */
static int isect(const double* T, const double x[3], const double v[3], double* t)
{
    const double p0 = v[1] * T[8] - v[2] * T[7];
    const double p1 = v[2] * T[6] - v[0] * T[8];
    const double p2 = v[0] * T[7] - v[1] * T[6];
    const double det = T[3] * p0 + T[4] * p1 + T[5] * p2;
    if (fabs(det) < 1e-14) return 0;
    const double inv = 1.0 / det;
    const double t0 = x[0] - T[0], t1 = x[1] - T[1], t2 = x[2] - T[2];
    const double u = (t0 * p0 + t1 * p1 + t2 * p2) * inv;
    if (u < 0.0 || u > 1.0) return 0;
    const double q0 = t1 * T[5] - t2 * T[4];
    const double q1 = t2 * T[3] - t0 * T[5];
    const double q2 = t0 * T[4] - t1 * T[3];
    const double w = (v[0] * q0 + v[1] * q1 + v[2] * q2) * inv;
    if (w < 0.0 || (u + w) > 1.0) return 0;
    *t = (T[6] * q0 + T[7] * q1 + T[8] * q2) * inv;
    return *t > 1e-14;
}

/* tryCachedCellIntersection, src/ProcessDSMC.cpp:1210-1251. The uncached
 * fallback (intersectFallbackCell, :1484-1524) evaluates the same products
 * on the same node coordinates and cannot find a hit this misses. */
static int find_exit(const OracleCase* o, int cell, int crossf, int prevTri, const double x[3], const double v[3],
                     double* tOut, int* triOut)
{
    double best = DBL_MAX;
    int bf = -2, bt = -1;
    for (int k = o->triOff[cell]; k < o->triOff[cell + 1]; ++k) {
        const int face = o->triFace[k], tag = o->triTag[k];
        if (face == crossf) {
            if (tag <= 0 || (prevTri != 1 && prevTri != 2) || tag == prevTri) continue;
        }
        double t = DBL_MAX;
        if (isect(&o->tri[(size_t)k * 9], x, v, &t) && t < best) { best = t; bf = face; bt = tag; }
    }
    *tOut = bf == -2 ? DBL_MAX : best;
    *triOut = bt;
    return bf;
}

typedef struct { int hitFace, hitTri, ncross; } TLog;

/* ParticleTransportOps::traceParticleDtleft + CrossboundarySwitch,
 * src/ProcessDSMC.cpp:149-221 and 1702-1829 */
static int trace(OracleCase* o, double x[3], double v[3], double* ir, int* cell, int crossf, int tag, double* dtleft,
                 Stream* rs, int istep, int stopWall, TLog* tlog)
{
    int ifout = T_STAY, iter = 0;
    while (*dtleft > 0.0) {
        if (iter++ >= o->maxCross) { o->ctr[K_LOST]++; *dtleft = 0.0; return T_LOST; }
        double t;
        int tri;
        const int face = find_exit(o, *cell, crossf, tag, x, v, &t, &tri);
        if (face == -2 || !isfinite(t) || t <= 0.0) { o->ctr[K_DROP]++; *dtleft = 0.0; return T_DROPPED; }
        if (t >= *dtleft) {
            for (int d = 0; d < 3; ++d) x[d] += v[d] * *dtleft;
            *dtleft = 0.0;
            return ifout;
        }
        crossf = face;
        tag = tri;
        const int role = o->role[face];
        if (tlog && role != R_INTERFACE && tlog->hitFace < 0) {
            tlog->hitFace = face;
            tlog->hitTri = tri;
            if (stopWall && role == R_WALL) {
                for (int d = 0; d < 3; ++d) x[d] += v[d] * t;
                *dtleft -= t;
                return ifout;
            }
        }
        o->ctr[K_CROSS]++;
        if (tlog) tlog->ncross++;
        if (role != R_NONE)
            for (int d = 0; d < 3; ++d) x[d] += v[d] * t;
        if (role == R_INTERFACE) {
            ifout = T_MOVED;
            *dtleft -= t;
            const int c0 = o->edges[face].faceMap[4], c1 = o->edges[face].faceMap[5];
            int next;
            if (*cell == c0) next = c1;
            else if (*cell == c1) next = c0;
            else next = c0;
            if (next < 0 || next >= o->ncell) { o->ctr[K_LOST]++; *dtleft = 0.0; return T_LOST; }
            *cell = next;
        } else if (role == R_INLET || role == R_OUTLET) {
            o->ctr[K_REM]++;
            *dtleft = 0.0;
            return T_REMOVED;
        } else if (role == R_WALL) {
            *dtleft -= t;
            const int w = o->faceWall[face];
            const double* R = &o->wallRot[(size_t)w * 18 + (tri == 2 ? 9 : 0)];
            const double v0 = v[0], v1 = v[1], v2 = v[2], ir0 = *ir;
            const double r1 = st_u64(rs), r2 = st_u64(rs), al = st_u64(rs), r3 = st_u64(rs);
            const double st = sqrt(o->m.Twall_ref);
            const double a = sqrt(-log(r2));
            const double vxp = a * sin(2.0 * M_PI * al) * st;
            const double vyp = a * cos(2.0 * M_PI * al) * st;
            const double vzp = -sqrt(-log(r1)) * st;
            v[0] = R[0] * vxp + R[1] * vyp + R[2] * vzp;
            v[1] = R[3] * vxp + R[4] * vyp + R[5] * vzp;
            v[2] = R[6] * vxp + R[7] * vyp + R[8] * vzp;
            *ir = -log(r3) * o->m.Twall_ref * 0.5;
            o->ctr[K_WALL]++;
            if (o->wallStats && istep > o->nss) {   /* recordBoundaryStressHeat, :1659-1689 */
                double* T = &o->wall[(size_t)w * 6];
                T[0] += 1.0;
                T[1] += v[0] - v0; T[2] += v[1] - v1; T[3] += v[2] - v2;
                T[4] += 0.5 * ((v[0] * v[0] + v[1] * v[1] + v[2] * v[2]) - (v0 * v0 + v1 * v1 + v2 * v2));
                T[5] += *ir - ir0;
            }
        } else if (role == R_SPECULAR) {
            *dtleft -= t;
            const int w = o->faceWall[face];
            const double* R = &o->wallRot[(size_t)w * 18 + (tri == 2 ? 9 : 0)];
            const double vn = v[0] * R[2] + v[1] * R[5] + v[2] * R[8];
            v[0] -= 2 * vn * R[2]; v[1] -= 2 * vn * R[5]; v[2] -= 2 * vn * R[8];
            o->ctr[K_WALL]++;
        }
    }
    return ifout;
}

void oracle_trace(OracleCase* o, int64_t n, const double* px, const double* py, const double* pz, const double* vx,
                  const double* vy, const double* vz, const double* dt, const int* cell, int stop_at_wall,
                  int* out_cell, int* out_ifout, int* out_face, int* out_tri, int* out_ncross, double* out_px,
                  double* out_py, double* out_pz, double* out_vx, double* out_vy, double* out_vz, double* out_dt)
{
    for (int64_t i = 0; i < n; ++i) {
        double x[3] = {px[i], py[i], pz[i]}, v[3] = {vx[i], vy[i], vz[i]}, ir = 0.0, dtl = dt[i];
        int c = cell[i];
        Stream rs;
        st_init(&rs, (uint32_t)i, 0u, 1u, o->k0, o->k1);
        TLog tl = {-1, 0, 0};
        const int out = trace(o, x, v, &ir, &c, -1, -1, &dtl, &rs, 0, stop_at_wall, &tl);
        out_cell[i] = out == T_REMOVED ? -1 : c;
        out_ifout[i] = out >= 0 ? out : -1;
        out_face[i] = tl.hitFace;
        out_tri[i] = tl.hitTri;
        out_ncross[i] = tl.ncross;
        out_px[i] = x[0]; out_py[i] = x[1]; out_pz[i] = x[2];
        out_vx[i] = v[0]; out_vy[i] = v[1]; out_vz[i] = v[2];
        out_dt[i] = dtl;
    }
}

/* ------------------------------------------------------------------------ */
/* particle store                                                            */
/* ------------------------------------------------------------------------ */
static int reserve(OracleCase* o, int64_t cap)
{
    if (cap <= o->cap) return 1;
    double** arrs[7] = {&o->px, &o->py, &o->pz, &o->vx, &o->vy, &o->vz, &o->ir};
    for (int k = 0; k < 7; ++k) {
        double* p = (double*)realloc(*arrs[k], sizeof(double) * (size_t)cap);
        if (!p) return 0;
        *arrs[k] = p;
    }
    int* q = (int*)realloc(o->pc, sizeof(int) * (size_t)cap);
    if (!q) return 0;
    o->pc = q;
    o->cap = cap;
    return 1;
}

int oracle_set_particles(OracleCase* o, int64_t n, const double* px, const double* py, const double* pz,
                         const double* vx, const double* vy, const double* vz, const double* ir, const int* cell)
{
    if (!reserve(o, n + 16)) return -3;
    memset(o->start, 0, sizeof(int) * ((size_t)o->ncell + 1));
    for (int64_t i = 0; i < n; ++i) {
        if (cell[i] < 0 || cell[i] >= o->ncell) return -1;
        o->start[cell[i] + 1]++;
    }
    for (int c = 0; c < o->ncell; ++c) o->start[c + 1] += o->start[c];
    int* fill = (int*)malloc(sizeof(int) * (size_t)o->ncell);
    memcpy(fill, o->start, sizeof(int) * (size_t)o->ncell);
    for (int64_t i = 0; i < n; ++i) {
        const int j = fill[cell[i]]++;
        o->px[j] = px[i]; o->py[j] = py[i]; o->pz[j] = pz[i];
        o->vx[j] = vx[i]; o->vy[j] = vy[i]; o->vz[j] = vz[i];
        o->ir[j] = ir[i]; o->pc[j] = cell[i];
    }
    free(fill);
    o->n = n;
    o->nInj = 0;
    o->sorted = 1;
    return 0;
}

int64_t oracle_count(const OracleCase* o) { return o->n; }

void oracle_get_particles(const OracleCase* o, double* px, double* py, double* pz, double* vx, double* vy, double* vz,
                          double* ir, int* cell)
{
    for (int64_t i = 0; i < o->n; ++i) {
        if (px) px[i] = o->px[i];
        if (py) py[i] = o->py[i];
        if (pz) pz[i] = o->pz[i];
        if (vx) vx[i] = o->vx[i];
        if (vy) vy[i] = o->vy[i];
        if (vz) vz[i] = o->vz[i];
        if (ir) ir[i] = o->ir[i];
        if (cell) cell[i] = o->pc[i];
    }
}

/* ------------------------------------------------------------------------ */
/* stages                                                                    */
/* ------------------------------------------------------------------------ */
/* preprocesseffquad, src/ProcessDSMC.cpp:2556-2570 with
 * emitParticlesFromBoundaryPatch :2501-2543, sampleBoundaryParticle
 * :2416-2458 and traceBoundaryParticle :2471-2488 */
static int inject(OracleCase* o, int istep)
{
    int total = 0;
    int* cnt = (int*)malloc(sizeof(int) * ((size_t)o->npatch + 1));
    for (int p = 0; p < o->npatch; ++p) {
        const int c = o->patches[p].cell;
        const double addNum = o->patches[p].addBase + o->remInj[c];
        const int n = (int)floor(addNum);
        o->remInj[c] = addNum - n;
        cnt[p] = n;
        total += n;
    }
    if (!reserve(o, o->n + total + 16)) { free(cnt); return -3; }
    int slot = 0;
    for (int p = 0; p < o->npatch; ++p) {
        const Patch* pt = &o->patches[p];
        for (int k = 0; k < cnt[p]; ++k, ++slot) {
            const int64_t gi = o->n + slot;
            Stream rs;
            st_init(&rs, (uint32_t)gi, (uint32_t)istep, 2u, o->k0, o->k1);
            double u = st_u64(&rs), w = st_u64(&rs);
            if (u + w > 1.0) { u = 1.0 - u; w = 1.0 - w; }
            double x[3];
            for (int d = 0; d < 3; ++d) x[d] = pt->geom[d] + u * pt->geom[3 + d] + w * pt->geom[6 + d];
            const double snp = pt->gas[0], fs1 = pt->gas[1], fs2 = pt->gas[2], stp1 = pt->gas[3], stp2 = pt->gas[4];
            const double tN = pt->gas[5], sq = pt->gas[6], QA = pt->gas[7];
            double vzr = 0.0, vza = 0.0;
            for (int outer = 0;; ++outer) {
                for (int inner = 0;; ++inner) {
                    const double r = st_u64(&rs);
                    vzr = (-QA + 2.0 * QA * r) * sq;
                    vza = vzr / sq + snp;
                    if (vza > 0) break;
                    if (inner > (1 << 20)) { vza = 1e-3; break; }
                }
                const double vzn = vzr / sq;
                const double pp = (2.0 * vza / fs1) * exp(fs2 - vzn * vzn);
                if (st_u64(&rs) < pp) break;
                if (outer > (1 << 20)) break;
            }
            const double r = st_u64(&rs), th = st_u64(&rs);
            const double a = sqrt(-log(r));
            const double vxa = (a * sin(2.0 * M_PI * th) + stp1) * sq;
            const double vya = (a * cos(2.0 * M_PI * th) + stp2) * sq;
            vza *= sq;
            const double* R = pt->rot;
            double v[3] = {R[0] * vxa + R[1] * vya + R[2] * vza, R[3] * vxa + R[4] * vya + R[5] * vza,
                           R[6] * vxa + R[7] * vya + R[8] * vza};
            double ir = -log(st_u64(&rs)) * tN * 0.5;
            double dtl = st_u64(&rs) * o->m.dtime;
            int c = pt->cell;
            const int out = trace(o, x, v, &ir, &c, pt->edge, pt->tag, &dtl, &rs, istep, 0, NULL);
            o->px[gi] = x[0]; o->py[gi] = x[1]; o->pz[gi] = x[2];
            o->vx[gi] = v[0]; o->vy[gi] = v[1]; o->vz[gi] = v[2];
            o->ir[gi] = ir;
            o->pc[gi] = out >= 0 ? c : -1;
        }
    }
    o->ctr[K_INJ] += (uint64_t)total;
    o->nInj = total;
    free(cnt);
    return 0;
}

/* advection, src/ProcessDSMC.cpp:1946-2017 */
static void move(OracleCase* o, int istep)
{
    for (int64_t i = 0; i < o->n; ++i) {
        double x[3] = {o->px[i], o->py[i], o->pz[i]}, v[3] = {o->vx[i], o->vy[i], o->vz[i]};
        double ir = o->ir[i], dtl = o->m.dtime;
        int c = o->pc[i];
        Stream rs;
        st_init(&rs, (uint32_t)i, (uint32_t)istep, 1u, o->k0, o->k1);
        const int out = trace(o, x, v, &ir, &c, -1, -1, &dtl, &rs, istep, 0, NULL);
        o->px[i] = x[0]; o->py[i] = x[1]; o->pz[i] = x[2];
        o->vx[i] = v[0]; o->vy[i] = v[1]; o->vz[i] = v[2];
        o->ir[i] = ir;
        o->pc[i] = out >= 0 ? c : -1;
    }
}

/* cache2chain, src/ProcessDSMC.cpp:2030-2135, in the canonical order: per
 * destination cell, arrivals grouped by where they come from (the cell
 * itself, then the neighbour across each of its faces in face order, then
 * everything else), each group in source order. */
static int sort_particles(OracleCase* o)
{
    const int64_t nt = o->n + o->nInj;
    int* key = (int*)malloc(sizeof(int) * (size_t)(nt + 1));
    int* cntk = (int*)calloc((size_t)o->ncell * 8 + 1, sizeof(int));
    /* source cell of each particle: from the layout before the move */
    int64_t kept = 0;
    for (int s = 0; s < o->ncell; ++s) {
        for (int i = o->start[s]; i < o->start[s + 1]; ++i) {
            const int d = o->pc[i];
            if (d < 0) { key[i] = -1; continue; }
            int slot = 7;
            if (d == s) slot = 0;
            else
                for (int j = 0; j < 6 && j < o->cells[s].num; ++j)
                    if (o->cells[s].cell2cell[j] == d) { slot = o->rev[(size_t)s * 6 + j] >= 0 ? o->rev[(size_t)s * 6 + j] + 1 : 7; break; }
            key[i] = d * 8 + slot;
        }
    }
    for (int64_t i = o->n; i < nt; ++i) key[i] = o->pc[i] < 0 ? -1 : o->pc[i] * 8 + 7;
    for (int64_t i = 0; i < nt; ++i)
        if (key[i] >= 0) { cntk[key[i] + 1]++; ++kept; }
    for (int k = 0; k < o->ncell * 8; ++k) cntk[k + 1] += cntk[k];
    double* nb[7];
    for (int k = 0; k < 7; ++k) nb[k] = (double*)malloc(sizeof(double) * (size_t)(kept + 16));
    int* nc = (int*)malloc(sizeof(int) * (size_t)(kept + 16));
    double* src[7] = {o->px, o->py, o->pz, o->vx, o->vy, o->vz, o->ir};
    for (int64_t i = 0; i < nt; ++i) {
        if (key[i] < 0) continue;
        const int j = cntk[key[i]]++;
        for (int k = 0; k < 7; ++k) nb[k][j] = src[k][i];
        nc[j] = key[i] >> 3;
    }
    for (int k = 0; k < 7; ++k) {
        free(src[k]);
    }
    o->px = nb[0]; o->py = nb[1]; o->pz = nb[2]; o->vx = nb[3]; o->vy = nb[4]; o->vz = nb[5]; o->ir = nb[6];
    free(o->pc);
    o->pc = nc;
    o->cap = kept + 16;
    o->n = kept;
    o->nInj = 0;
    memset(o->start, 0, sizeof(int) * ((size_t)o->ncell + 1));
    for (int64_t i = 0; i < kept; ++i) o->start[nc[i] + 1]++;
    for (int c = 0; c < o->ncell; ++c) o->start[c + 1] += o->start[c];
    free(key);
    free(cntk);
    return 0;
}

static double collision_diameter(const OracleCase* o, double cr)   /* src/ProcessDSMC.cpp:2603-2608 */
{
    const double cr2 = cr * cr;
    return cr * o->cdPrefactor * pow(1.0 / cr2, o->m.eta);
}

/* collisionDSMC + collisionVelocity, src/ProcessDSMC.cpp:2621-2744 */
static void collide(OracleCase* o, int istep)
{
    for (int c = 0; c < o->ncell; ++c) {
        const int s0 = o->start[c];
        const int n = o->start[c + 1] - s0;
        if (n <= 1) continue;
        double crm = o->crmax[c];
        const double S = o->cells[c].area;
        const double consCrm = collision_diameter(o, crm * o->m.v_rms);
        const double pairs = 0.5 * n * (n - 1) * o->m.Neff * consCrm * o->m.dtime * o->m.dt_ref / S + o->remColl[c];
        const int npairs = (int)floor(pairs);
        o->remColl[c] = pairs - npairs;
        o->ctr[K_PAIRS] += (uint64_t)npairs;
        if (!(consCrm > 0.0)) continue;
        double* vx = o->vx + s0;
        double* vy = o->vy + s0;
        double* vz = o->vz + s0;
        double* ir = o->ir + s0;
        const double expLB = 1.0 / (2.5 - o->m.omega);
        for (int j = 0; j < npairs; ++j) {
            Stream rs;
            st_init(&rs, (uint32_t)c, (uint32_t)istep, 3u | ((uint32_t)j << 4), o->k0, o->k1);
            const int k1 = (int)mulhi(st_next(&rs), (uint32_t)n);
            int k2 = k1 + 1 + (int)mulhi(st_next(&rs), (uint32_t)(n - 1));
            if (k2 >= n) k2 -= n;
            const double vr0 = vx[k1] - vx[k2], vr1 = vy[k1] - vy[k2], vr2 = vz[k1] - vz[k2];
            const double cr2 = vr0 * vr0 + vr1 * vr1 + vr2 * vr2;
            const double cr = sqrt(cr2);
            double preErt = 0.5 * 0.5 * cr2;
            if (cr > crm) crm = cr;
            const double accept = collision_diameter(o, cr * o->m.v_rms) / consCrm;
            if (st_u64(&rs) >= accept) continue;
            /* the relaxation test's variate and the energy fraction's are
             * both drawn for each particle whether or not it relaxes, so an
             * accepted pair always reads the same stream positions */
            for (int h = 0; h < 2; ++h) {
                double* irp = h == 0 ? &ir[k1] : &ir[k2];
                const double u = st_u64(&rs);
                const double r = st_u64(&rs);
                if (u <= o->m.P_relax) {
                    const double preEr = *irp;
                    const double postEr = (preErt + preEr) * (1.0 - pow(r, expLB));
                    *irp = postEr;
                    preErt = preErt + preEr - postEr;
                }
            }
            const double postVr = sqrt(2.0 * preErt / 0.5);
            const double vc0 = 0.5 * (vx[k1] + vx[k2]), vc1 = 0.5 * (vy[k1] + vy[k2]), vc2 = 0.5 * (vz[k1] + vz[k2]);
            const double r = st_u64(&rs);
            const double cosChi = 2.0 * pow(r, 1.0 / o->m.alpha) - 1.0;
            const double sinChi = sqrt(1.0 - cosChi * cosChi);
            const double th = st_u64(&rs);
            const double sth = sin(2.0 * M_PI * th), cth = cos(2.0 * M_PI * th);
            const double vrp = sqrt(vr1 * vr1 + vr2 * vr2);
            const double scale = postVr / (cr > 1.0e-300 ? cr : 1.0e-300);
            const double vrpc = vrp > 1.0e-300 ? vrp : 1.0e-300;
            double r1 = scale * (cosChi * vr0 + sinChi * sth * vrp);
            double r2 = scale * (cosChi * vr1 + sinChi * (cr * vr2 * cth - vr0 * vr1 * sth) / vrpc);
            double r3 = scale * (cosChi * vr2 - sinChi * (cr * vr1 * cth + vr0 * vr2 * sth) / vrpc);
            if (vrp < 1e-6) {
                r1 = scale * cosChi * vr0;
                r2 = scale * sinChi * vr0 * cth;
                r3 = scale * sinChi * vr0 * sth;
            }
            vx[k1] = vc0 + 0.5 * r1; vy[k1] = vc1 + 0.5 * r2; vz[k1] = vc2 + 0.5 * r3;
            vx[k2] = vc0 - 0.5 * r1; vy[k2] = vc1 - 0.5 * r2; vz[k2] = vc2 - 0.5 * r3;
            o->ctr[K_COLL]++;
        }
        o->crmax[c] = crm;
    }
}

/* writeAveragedMacro + guardInvalidMacro, src/ProcessDSMC.cpp:3126-3211;
 * writeLocalMacro / writeRecordMacro, :3224-3299 */
static void macro_core(const double* m, double Np, double rho, double dr, double* out)
{
    out[0] = rho;
    out[1] = m[1] / Np; out[2] = m[2] / Np; out[3] = m[3] / Np;
    const double ux = out[1], uy = out[2], uz = out[3];
    const double ux2 = ux * ux, uy2 = uy * uy, uz2 = uz * uz;
    const double u2 = ux2 + uy2 + uz2;
    out[4] = 2.0 / 3.0 / Np * (m[4] - Np * u2);
    const double T = out[4];
    out[5] = 2.0 * rho / Np * (2.0 / 3.0 * m[5] - 1.0 / 3.0 * m[7] - 1.0 / 3.0 * m[9] - 2.0 / 3.0 * Np * ux2 + 1.0 / 3.0 * Np * uy2 + 1.0 / 3.0 * Np * uz2);
    out[6] = 2.0 * rho / Np * (m[6] - Np * ux * uy);
    out[7] = 2.0 * rho / Np * (2.0 / 3.0 * m[7] - 1.0 / 3.0 * m[5] - 1.0 / 3.0 * m[9] - 2.0 / 3.0 * Np * uy2 + 1.0 / 3.0 * Np * ux2 + 1.0 / 3.0 * Np * uz2);
    out[8] = 2.0 * rho / Np * (m[8] - Np * uy * uz);
    out[9] = 2.0 * rho / Np * (2.0 / 3.0 * m[9] - 1.0 / 3.0 * m[5] - 1.0 / 3.0 * m[7] - 2.0 / 3.0 * Np * uz2 + 1.0 / 3.0 * Np * ux2 + 1.0 / 3.0 * Np * uy2);
    out[10] = 2.0 * rho / Np * (m[10] - Np * uz * ux);
    out[11] = rho / Np * (m[11] - 2 * ux * m[5] - 2 * uy * m[6] - 2 * uz * m[10] + u2 * m[1]) - ux * 1.5 * T * rho;
    out[12] = rho / Np * (m[12] - 2 * ux * m[6] - 2 * uy * m[7] - 2 * uz * m[8] + u2 * m[2]) - uy * 1.5 * T * rho;
    out[13] = rho / Np * (m[13] - 2 * ux * m[10] - 2 * uy * m[8] - 2 * uz * m[9] + u2 * m[3]) - uz * 1.5 * T * rho;
    out[14] = 4.0 / dr / Np * m[14];
    out[15] = 2.0 * rho / Np * (m[15] - ux * m[14]);
    out[16] = 2.0 * rho / Np * (m[16] - uy * m[14]);
    out[17] = 2.0 * rho / Np * (m[17] - uz * m[14]);
}

static void averaged(const OracleCase* o, const double* m, double count, double S, double* out)
{
    const double Np = m[0];
    if (!(Np > 1.0e-12) || !isfinite(Np) || !(count > 0.0) || !isfinite(count) || !(S > 0.0) || !isfinite(S) ||
        !(o->m.Neff > 0.0) || !isfinite(o->m.Neff) || !(o->m.n_ref > 0.0) || !isfinite(o->m.n_ref) ||
        !(o->m.dr > 0.0) || !isfinite(o->m.dr)) {
        for (int j = 0; j < 18; ++j) out[j] = 0.0;
        return;
    }
    macro_core(m, Np, o->m.Neff / S * Np / count / o->m.n_ref, o->m.dr, out);
    int valid = (out[0] > 0.0) && isfinite(out[0]) && (out[4] > 0.0) && isfinite(out[4]) && (out[14] > 0.0) &&
                isfinite(out[14]);
    for (int j = 0; valid && j < 18; ++j) valid = isfinite(out[j]);
    if (!valid)
        for (int j = 0; j < 18; ++j) out[j] = 0.0;
}

/* accumulateCellMoments, src/ProcessDSMC.cpp:2951-3006 */
static void moments(const OracleCase* o, int c, double m[18])
{
    for (int k = 0; k < 18; ++k) m[k] = 0.0;
    for (int i = o->start[c]; i < o->start[c + 1]; ++i) {
        const double x = o->vx[i], y = o->vy[i], z = o->vz[i], I = o->ir[i];
        const double v2 = x * x + y * y + z * z;
        m[0] += 1.0; m[1] += x; m[2] += y; m[3] += z; m[4] += v2;
        m[5] += x * x; m[6] += x * y; m[7] += y * y; m[8] += y * z; m[9] += z * z; m[10] += z * x;
        m[11] += x * v2; m[12] += y * v2; m[13] += z * v2;
        m[14] += I; m[15] += x * I; m[16] += y * I; m[17] += z * I;
    }
}

/* statistic_macro, src/ProcessDSMC.cpp:2757-2861 */
static void sample(OracleCase* o, int istep)
{
    const int every = (istep % o->nevery) == 0;
    const int ngsis = o->nevery * o->nrepeat;
    for (int c = 0; c < o->ncell; ++c) {
        double m[18];
        moments(o, c, m);
        memcpy(&o->stepMom[(size_t)c * 18], m, sizeof m);
        double* acc = &o->acc[(size_t)c * 54];
        const double na = (double)o->nscheme;
        const double w = (istep <= o->nscheme) ? 1.0 : (na - 1.0) / na;
        for (int k = 0; k < 18; ++k) {
            if (w == 1.0) acc[k] += m[k];
            else acc[k] = w * acc[k] + m[k];
            if (istep > o->nss) acc[18 + k] += m[k];
            if (every) acc[36 + k] += m[k];
        }
        if (every && (o->sparse[c] == 1 || o->sparse[c] == 2)) {
            if (o->saccum[c] < 0) o->saccum[c] = 0;
            ++o->saccum[c];
        }
        if (ngsis > 0 && istep % ngsis == 0) {
            const double* inter = acc + 36;
            const double ws = inter[0];
            const int finite = isfinite(ws);
            int sparse = (o->sparse[c] == 1 || o->sparse[c] == 2);
            if (!sparse && finite && ws < 3.0) {
                o->sparse[c] = 1;
                o->saccum[c] = o->nrepeat > 1 ? o->nrepeat : 1;
                sparse = 1;
            }
            const int valid = (ws >= 3.0) && finite;
            o->wsamp[c] = ws;
            o->wvalid[c] = (char)valid;
            const double S = o->cells[c].area;
            if (sparse) averaged(o, inter, (double)(o->saccum[c] > 1 ? o->saccum[c] : 1), S, &o->record[(size_t)c * 18]);
            else if (valid) averaged(o, inter, (double)o->nrepeat, S, &o->record[(size_t)c * 18]);
            if (!sparse)
                for (int k = 0; k < 18; ++k) acc[36 + k] = 0.0;
        }
    }
    o->localLazy = 1;
    o->lastIstep = istep;
}

void oracle_macro_pre(OracleCase* o)   /* statistic_macroPre, src/ProcessDSMC.cpp:3312-3326 */
{
    for (int c = 0; c < o->ncell; ++c) {
        double m[18];
        moments(o, c, m);
        memcpy(&o->stepMom[(size_t)c * 18], m, sizeof m);
        const double S = o->cells[c].area;
        double* L = &o->local[(size_t)c * 18];
        if (!(m[0] > 0.0) || !isfinite(m[0])) {
            for (int k = 0; k < 18; ++k) L[k] = 0.0;
        } else {
            macro_core(m, m[0], o->m.Neff / S * m[0] / o->m.n_ref, o->m.dr, L);
        }
        macro_core(m, m[0], o->m.Neff / S * m[0] / o->m.n_ref, o->m.dr, &o->record[(size_t)c * 18]);
    }
    o->localLazy = 0;
}

int oracle_step(OracleCase* o, int istep, unsigned stages)
{
    if (stages & 1u) {
        const int r = inject(o, istep);
        if (r) return r;
    }
    if (stages & 2u) move(o, istep);
    if (stages & 4u) sort_particles(o);
    if (stages & 8u) collide(o, istep);
    if (stages & 16u) sample(o, istep);
    return 0;
}

void oracle_get_macro(OracleCase* o, int which, double* out)
{
    const size_t nc = (size_t)o->ncell;
    if (which == 0) {
        if (o->localLazy)
            for (size_t c = 0; c < nc; ++c) averaged(o, &o->acc[c * 54], (double)o->nscheme, o->cells[c].area, &o->local[c * 18]);
        memcpy(out, o->local, sizeof(double) * nc * 18);
    } else if (which == 1) {
        memcpy(out, o->record, sizeof(double) * nc * 18);
    } else {
        if (o->lastIstep > o->nss)
            for (size_t c = 0; c < nc; ++c)
                averaged(o, &o->acc[c * 54 + 18], (double)(o->lastIstep - o->nss), o->cells[c].area, &o->finalRecord[c * 18]);
        memcpy(out, o->finalRecord, sizeof(double) * nc * 18);
    }
}

void oracle_get_step_moments(const OracleCase* o, double* out)
{
    memcpy(out, o->stepMom, sizeof(double) * (size_t)o->ncell * 18);
}

void oracle_get_acc(const OracleCase* o, double* out) { memcpy(out, o->acc, sizeof(double) * (size_t)o->ncell * 54); }

void oracle_get_cell_state(const OracleCase* o, double* crmax, double* rem_coll, double* rem_inj)
{
    const size_t b = sizeof(double) * (size_t)o->ncell;
    if (crmax) memcpy(crmax, o->crmax, b);
    if (rem_coll) memcpy(rem_coll, o->remColl, b);
    if (rem_inj) memcpy(rem_inj, o->remInj, b);
}

void oracle_set_cell_state(OracleCase* o, const double* crmax, const double* rem_coll, const double* rem_inj)
{
    const size_t b = sizeof(double) * (size_t)o->ncell;
    if (crmax) memcpy(o->crmax, crmax, b);
    if (rem_coll) memcpy(o->remColl, rem_coll, b);
    if (rem_inj) memcpy(o->remInj, rem_inj, b);
}

int oracle_set_sparse_state(OracleCase* o, const unsigned char* sparse_state)
{
    for (int c = 0; c < o->ncell; ++c)
        if (sparse_state[c] > 2) return -1;
    memcpy(o->sparse, sparse_state, (size_t)o->ncell);
    return 0;
}

void oracle_get_counts(const OracleCase* o, int* ppc, double* window_samples, char* window_valid,
                       unsigned char* sparse_state)
{
    for (int c = 0; c < o->ncell; ++c) {
        if (ppc) ppc[c] = o->start[c + 1] - o->start[c];
        if (window_samples) window_samples[c] = o->wsamp[c];
        if (window_valid) window_valid[c] = o->wvalid[c];
        if (sparse_state) sparse_state[c] = o->sparse[c];
    }
}

void oracle_get_wall(const OracleCase* o, double* tally)
{
    memset(tally, 0, sizeof(double) * (size_t)o->nface * 6);
    for (int f = 0; f < o->nface; ++f)
        if (o->faceWall[f] >= 0 && o->role[f] == R_WALL)
            memcpy(&tally[(size_t)f * 6], &o->wall[(size_t)o->faceWall[f] * 6], sizeof(double) * 6);
}

void oracle_counters(const OracleCase* o, uint64_t out[8]) { memcpy(out, o->ctr, sizeof(uint64_t) * 8); }

/* ------------------------------------------------------------------------ */
/* placement tetrahedra, initial fill and the GSIS particle update           */
/* ------------------------------------------------------------------------ */
static double philox_u64(uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, uint32_t k0, uint32_t k1, int half)
{
    const uint32_t c[4] = {c0, c1, c2, c3}, k[2] = {k0, k1};
    uint32_t out[4];
    oracle_philox(c, k, out);
    const uint64_t a = half ? out[2] : out[0], b = half ? out[3] : out[1];
    const uint64_t q = (a << 21) ^ (b >> 11);
    return ((double)q + 0.5) * 0x1.0p-53;
}

/* |(P1-P0) . ((P2-P0) x (P3-P0))| / 6: tetAbsVolume and appendCenterFaceTet,
 * src/ProcessGSIS.cpp:660-675, 829-870 */
static double tet_volume(const double* P0, const double* P1, const double* P2, const double* P3)
{
    const double ax = P1[0] - P0[0], ay = P1[1] - P0[1], az = P1[2] - P0[2];
    const double bx = P2[0] - P0[0], by = P2[1] - P0[1], bz = P2[2] - P0[2];
    const double cx = P3[0] - P0[0], cy = P3[1] - P0[1], cz = P3[2] - P0[2];
    const double crx = by * cz - bz * cy, cry = bz * cx - bx * cz, crz = bx * cy - by * cx;
    return fabs(ax * crx + ay * cry + az * crz) / 6.0;
}

static int node_ok(const OracleCase* o, int n) { return n >= 0 && n < o->npoint; }

/* one tetrahedron: vertices V0 (the centre when ctr != NULL) and nodes */
static int place_add(const OracleCase* o, const double* ctr, const int* nodes, double* V, double* vol, int* nt)
{
    double* v = V + (size_t)(*nt) * 12;
    int k0 = 0;
    if (ctr) { v[0] = ctr[0]; v[1] = ctr[1]; v[2] = ctr[2]; k0 = 1; }
    for (int k = k0; k < 4; ++k) {
        const int n = nodes[k - k0];
        if (!node_ok(o, n)) return 0;
        memcpy(v + 3 * k, o->pts + (size_t)n * 3, 3 * sizeof(double));
    }
    const double w = tet_volume(v, v + 3, v + 6, v + 9);
    if (!(w > 0.0) || !isfinite(w)) return 0;
    vol[*nt] = w;
    ++*nt;
    return 1;
}

/* buildCellInitTets (src/MeshparticalInitial.cpp:172-355, the same
 * decomposition as src/ProcessGSIS.cpp:748-964) for cell c: appendTetCellTets,
 * then appendPyramidCellTets, then appendCenterFaceTets. V gets 12 doubles
 * and vol one per tetrahedron (room for 12). Returns the number (0: none). */
static int place_cell(const OracleCase* o, int c, double* V, double* vol)
{
    const Cell* cl = &o->cells[c];
    const int nf = cl->num < 6 ? cl->num : 6;
    int uniq[24], nu = 0, nodesOk = 1;
    for (int m = 0; m < nf && nodesOk; ++m) {
        const int f = cl->cell2face[m];
        if (f < 0 || f >= o->nface) { nodesOk = 0; break; }
        const Edge* e = &o->edges[f];
        if (e->faceType != 3 && e->faceType != 4) { nodesOk = 0; break; }
        for (int k = 0; k < e->faceType; ++k) {
            const int n = e->faceMap[k];
            if (!node_ok(o, n)) { nodesOk = 0; break; }
            int seen = 0;
            for (int q = 0; q < nu; ++q) seen |= uniq[q] == n;
            if (!seen) uniq[nu++] = n;
        }
    }
    int nt = 0;
    if (nodesOk && nu == 4 && place_add(o, NULL, uniq, V, vol, &nt)) return nt;
    nt = 0;
    int quad = -1, ok = 1;
    for (int m = 0; m < nf; ++m) {
        const int f = cl->cell2face[m];
        if (f < 0 || f >= o->nface) { ok = 0; break; }
        if (o->edges[f].faceType == 4) {
            if (quad >= 0) { ok = 0; break; }
            quad = f;
        }
    }
    if (ok && quad >= 0 && nodesOk && nu == 5) {
        const Edge* b = &o->edges[quad];
        int apex = -1;
        for (int q = 0; q < nu && apex < 0; ++q) {
            int on = 0;
            for (int k = 0; k < 4; ++k) on |= b->faceMap[k] == uniq[q];
            if (!on) apex = uniq[q];
        }
        if (apex >= 0) {
            int t0[3], t1[3];
            decode_split(o->split ? o->split[quad] : 0, t0, t1);
            if (t0[0] < 0 || t1[0] < 0) decode_split(0, t0, t1);
            const int a[4] = {b->faceMap[t0[0]], b->faceMap[t0[1]], b->faceMap[t0[2]], apex};
            const int d[4] = {b->faceMap[t1[0]], b->faceMap[t1[1]], b->faceMap[t1[2]], apex};
            if (place_add(o, NULL, a, V, vol, &nt) && place_add(o, NULL, d, V, vol, &nt)) return nt;
        }
    }
    nt = 0;
    for (int m = 0; m < nf; ++m) {
        const int f = cl->cell2face[m];
        if (f < 0 || f >= o->nface) return 0;
        const Edge* e = &o->edges[f];
        if (e->faceType == 3) {
            if (!place_add(o, cl->cellXY, e->faceMap, V, vol, &nt)) return 0;
        } else if (e->faceType == 4) {
            int t0[3], t1[3];
            decode_split(o->split ? o->split[f] : 0, t0, t1);
            if (t0[0] < 0 || t1[0] < 0) decode_split(0, t0, t1);
            const int a[3] = {e->faceMap[t0[0]], e->faceMap[t0[1]], e->faceMap[t0[2]]};
            const int d[3] = {e->faceMap[t1[0]], e->faceMap[t1[1]], e->faceMap[t1[2]]};
            if (!place_add(o, cl->cellXY, a, V, vol, &nt) || !place_add(o, cl->cellXY, d, V, vol, &nt)) return 0;
        } else {
            return 0;
        }
    }
    return nt;
}

int oracle_placement(const OracleCase* o, int* off, double* V, double* vol)
{
    double v[12 * 12], w[12];
    int n = 0;
    for (int c = 0; c < o->ncell; ++c) {
        const int nt = place_cell(o, c, v, w);
        if (off) off[c] = n;
        if (V) memcpy(V + (size_t)n * 12, v, sizeof(double) * 12 * (size_t)nt);
        if (vol) memcpy(vol + n, w, sizeof(double) * (size_t)nt);
        n += nt;
    }
    if (off) off[o->ncell] = n;
    return n;
}

/* randomBarycentric4 (src/MeshparticalInitial.cpp:85-106): four uniforms
 * over their sum; the point a V0 + b V1 + c V2 + d V3 */
static void place_point(const double* V, double r0, double r1, double r2, double r3, double out[3])
{
    const double sum = r0 + r1 + r2 + r3;
    double a = 0.25, b = 0.25, c = 0.25, d = 0.25;
    if (sum > 0.0 && isfinite(sum)) { a = r0 / sum; b = r1 / sum; c = r2 / sum; d = r3 / sum; }
    for (int k = 0; k < 3; ++k) out[k] = a * V[k] + b * V[3 + k] + c * V[6 + k] + d * V[9 + k];
}

/* sampleCellLocation (src/ProcessGSIS.cpp:977-1029) with randomlocation's
 * fallback to the cell centre (:2478-2488) */
static void place_in_cell(const OracleCase* o, int c, double uPick, double r0, double r1, double r2, double r3,
                          double out[3])
{
    double V[12 * 12], vol[12];
    const int nt = place_cell(o, c, V, vol);
    double total = 0.0;
    for (int t = 0; t < nt; ++t) total += vol[t];
    if (nt == 0 || !(total > 0.0) || !isfinite(total)) {
        memcpy(out, o->cells[c].cellXY, 3 * sizeof(double));
        return;
    }
    double pick = uPick * total;
    int ch = nt - 1;
    for (int t = 0; t < nt; ++t) {
        if (pick <= vol[t]) { ch = t; break; }
        pick -= vol[t];
    }
    place_point(V + (size_t)ch * 12, r0, r1, r2, r3, out);
}

/* Np_tri_inititial + adjust_particles (src/MeshparticalInitial.cpp:481-514,
 * 752-786) with Philox draws (c, t, 4, 1) for tetrahedron t's rounding and
 * (c, i, 4, 2) for shuffle step i; first[t] = the tetrahedron's first
 * particle. Returns the cell's count. */
static int fill_cell_counts(int c, int np, const double* vol, int nt, uint32_t k0, uint32_t k1, int* first)
{
    double region[12];
    int ind[12];
    if (np <= 0 || nt <= 0) {
        for (int t = 0; t < nt; ++t) first[t] = 0;
        return 0;
    }
    double sumVol = 0.0;
    for (int t = 0; t < nt; ++t) sumVol += vol[t];
    int sumN = 0;
    for (int t = 0; t < nt; ++t) {
        const double x = (double)np * vol[t] / sumVol;
        const double fl = floor(x);
        region[t] = (philox_u64((uint32_t)c, (uint32_t)t, 4u, 1u, k0, k1, 0) < x - fl) ? fl + 1.0 : fl;
        sumN += (int)region[t];
    }
    const int delta = np - sumN;
    const int ad = delta < 0 ? -delta : delta;
    const double stepv = delta > 0 ? 1.0 : -1.0;
    if (ad >= nt) {
        for (int t = 0; t < nt; ++t) region[t] += stepv;
    } else if (ad > 0) {
        for (int t = 0; t < nt; ++t) ind[t] = t;
        for (int i = 0; i < ad; ++i) {
            int r = i + (int)(philox_u64((uint32_t)c, (uint32_t)i, 4u, 2u, k0, k1, 0) * (double)(nt - i));
            if (r > nt - 1) r = nt - 1;
            const int tmp = ind[i]; ind[i] = ind[r]; ind[r] = tmp;
        }
        for (int i = 0; i < ad; ++i) region[ind[i]] += stepv;
    }
    int n = 0;
    for (int t = 0; t < nt; ++t) {
        first[t] = n;
        n += (int)(region[t] > 0.0 ? region[t] : 0.0);
    }
    return n;
}

int oracle_fill(OracleCase* o, double ppc_mean, uint64_t seed, int at_rest)
{
    const uint32_t k0 = (uint32_t)(seed & 0xffffffffu), k1 = (uint32_t)(seed >> 32);
    double vtot = 0.0;
    for (int c = 0; c < o->ncell; ++c) vtot += o->cells[c].area;
    if (!(vtot > 0.0) || !(ppc_mean > 0.0)) return -1;
    const double nps = ppc_mean * (double)o->ncell;
    double u[3] = {0.0, 0.0, 0.0}, sig = 1.0, tN = 1.0;
    if (!at_rest) {
        const Mess* m = &o->m;
        const double base = 1.0 * m->Ma * sqrt(m->gamma / 2.0) * m->v_in / m->v_rms;
        u[0] = base * o->dirx;
        u[1] = base * o->diry;
        tN = m->T_in / m->T_ref;
        sig = sqrt(tN / 2.0);
    }
    /* counts */
    int* cnt = (int*)malloc(sizeof(int) * (size_t)o->ncell);
    int* firsts = (int*)malloc(sizeof(int) * (size_t)o->ncell * 12);
    int64_t total = 0;
    double V[12 * 12], vol[12];
    for (int c = 0; c < o->ncell; ++c) {
        const double ns = o->cells[c].area * nps / vtot;
        const double fl = floor(ns);
        const int np = (int)fl + ((philox_u64((uint32_t)c, 0u, 4u, 0u, k0, k1, 0) < ns - fl) ? 1 : 0);
        const int nt = place_cell(o, c, V, vol);
        cnt[c] = fill_cell_counts(c, np, vol, nt, k0, k1, firsts + (size_t)c * 12);
        total += cnt[c];
    }
    if (!reserve(o, total + 16)) { free(cnt); free(firsts); return -3; }
    o->start[0] = 0;
    for (int c = 0; c < o->ncell; ++c) o->start[c + 1] = o->start[c] + cnt[c];
    for (int c = 0; c < o->ncell; ++c) {
        const int nt = place_cell(o, c, V, vol);
        const int* first = firsts + (size_t)c * 12;
        for (int k = 0; k < cnt[c]; ++k) {
            int t = 0;
            for (int q = 1; q < nt; ++q)
                if (first[q] <= k) t = q;
            double r[10];
            for (int b = 0; b < 5; ++b) {
                r[2 * b] = philox_u64((uint32_t)c, (uint32_t)k, 5u, (uint32_t)b, k0, k1, 0);
                r[2 * b + 1] = philox_u64((uint32_t)c, (uint32_t)k, 5u, (uint32_t)b, k0, k1, 1);
            }
            /* velocityLocationGenerate, src/MeshparticalInitial.cpp:646-721 */
            const double rad1 = sqrt(-2.0 * log(r[0])), th1 = 2 * M_PI * r[1];
            const double rad2 = sqrt(-2.0 * log(r[2])), th2 = 2 * M_PI * r[3];
            const int64_t j = o->start[c] + k;
            double x[3];
            place_point(V + (size_t)t * 12, r[5], r[6], r[7], r[8], x);
            o->px[j] = x[0]; o->py[j] = x[1]; o->pz[j] = x[2];
            o->vx[j] = u[0] + sig * (rad1 * sin(th1));
            o->vy[j] = u[1] + sig * (rad1 * cos(th1));
            o->vz[j] = u[2] + sig * (rad2 * sin(th2));
            o->ir[j] = -log(r[4]) * tN * 0.5;
            o->pc[j] = c;
        }
    }
    free(cnt);
    free(firsts);
    o->n = total;
    o->nInj = 0;
    o->sorted = 1;
    return 0;
}

/* molecular_velocity_change with replication, deletion, MaxwellianSample and
 * randomlocation (src/ProcessGSIS.cpp:2239-2530). The reference's mt19937
 * and rand() draws are replaced by Philox counters (cell, j, 6 | sub << 4 |
 * epoch << 8, block) under the case's seed: sub 0 the count rounding, 1 the
 * deletion draws (two per block), 2 the copies (choice, pick, 4 weights),
 * 3 the Maxwellian samples (3 x (r, th), (r, pick), 4 weights). Particles
 * are rebuilt cell by cell in the reference's bucket order. report: nan
 * cell (-1 none), cells updated, cells skipped, added, removed, particles.
 * Returns -2 (particles untouched) if a count falls outside [0, 2^30). */
int oracle_molecular_velocity_change(OracleCase* o, const double* ns, const char* accepted, int64_t report[6])
{
    const int ncell = o->ncell;
    const uint32_t P = 6u | ((o->gsisEpoch & 0xffffffu) << 8);
    int firstNan = ncell;
    for (int c = 0; c < ncell && firstNan == ncell; ++c) {
        if (accepted && accepted[c] == 0) continue;
        const double* r = ns + (size_t)c * 6;
        if (isnan(r[0]) || isnan(r[1]) || isnan(r[2]) || isnan(r[3])) firstNan = c;
    }
    int* target = (int*)malloc(sizeof(int) * (size_t)ncell);
    char* upd = (char*)calloc((size_t)ncell, 1);
    int64_t updated = 0, skipped = 0, added = 0, removed = 0, total = 0;
    for (int c = 0; c < ncell; ++c) {
        const int n0 = o->start[c + 1] - o->start[c];
        target[c] = n0;
        if (c < firstNan) {
            if (accepted && accepted[c] == 0) {
                ++skipped;
            } else {
                upd[c] = 1;
                ++updated;
                const double* r = ns + (size_t)c * 6;
                /* n_ns = nsresult * (area * n_ref) / Neff, Iround
                 * (src/MeshparticalInitial.cpp:730-742) */
                const double x = r[0] * (o->cells[c].area * o->m.n_ref) / o->m.Neff;
                const double fl = floor(x);
                const double nns = (philox_u64((uint32_t)c, 0u, P, 0u, o->k0, o->k1, 0) < x - fl) ? fl + 1.0 : fl;
                if (nns > (double)n0) {
                    if (!(nns < 1073741824.0)) { free(target); free(upd); return -2; }
                    if (!(n0 == 0 && r[4] < 0.0)) target[c] = (int)nns;
                } else if (nns < (double)n0 && nns >= 0.0) {
                    target[c] = (int)nns;
                }
            }
        }
        if (target[c] > n0) added += target[c] - n0;
        else removed += n0 - target[c];
        total += target[c];
    }
    double *nx = (double*)malloc(sizeof(double) * (size_t)(total + 1)), *ny = (double*)malloc(sizeof(double) * (size_t)(total + 1)),
           *nz = (double*)malloc(sizeof(double) * (size_t)(total + 1)), *nvx = (double*)malloc(sizeof(double) * (size_t)(total + 1)),
           *nvy = (double*)malloc(sizeof(double) * (size_t)(total + 1)), *nvz = (double*)malloc(sizeof(double) * (size_t)(total + 1)),
           *nir = (double*)malloc(sizeof(double) * (size_t)(total + 1));
    int* npc = (int*)malloc(sizeof(int) * (size_t)(total + 1));
    int* nstart = (int*)malloc(sizeof(int) * ((size_t)ncell + 1));
    nstart[0] = 0;
    for (int c = 0; c < ncell; ++c) nstart[c + 1] = nstart[c] + target[c];
    int cap = 64;
    int* perm = (int*)malloc(sizeof(int) * (size_t)cap);
    for (int c = 0; c < ncell; ++c) {
        const int sA = o->start[c], n0 = o->start[c + 1] - sA;
        const int sB = nstart[c], n1 = target[c];
        const int need = (n0 > n1 ? n0 : n1) + 1;
        if (need > cap) { cap = need; perm = (int*)realloc(perm, sizeof(int) * (size_t)cap); }
        /* perm[q]: the old particle at bucket position q (copies: the original) */
        for (int k = 0; k < n0; ++k) perm[k] = k;
        const double* r = ns + (size_t)c * 6;
        int sampled = 0;
        if (n1 < n0) {
            for (int j = 0; j < n0 - n1; ++j) {   /* deletion, src/ProcessGSIS.cpp:2490-2530 */
                const int m = n0 - j;
                int kp = (int)(philox_u64((uint32_t)c, (uint32_t)(j >> 1), P | (1u << 4), 0u, o->k0, o->k1, j & 1) * (double)m);
                if (kp > m - 1) kp = m - 1;
                perm[kp] = perm[m - 1];
            }
        } else if (n1 > n0 && n0 > 0) {
            for (int j = 0; j < n1 - n0; ++j) {   /* replication, src/ProcessGSIS.cpp:2368-2441 */
                const int m = n0 + j;
                int kp = (int)(philox_u64((uint32_t)c, (uint32_t)j, P | (2u << 4), 0u, o->k0, o->k1, 0) * (double)m);
                if (kp > m - 1) kp = m - 1;
                perm[n0 + j] = perm[kp];
            }
        } else if (n1 > n0) {
            sampled = 1;
        }
        for (int q = 0; q < n1; ++q) {
            const int64_t to = sB + q;
            npc[to] = c;
            if (sampled) {   /* MaxwellianSample, src/ProcessGSIS.cpp:2443-2466 */
                double w[12];
                for (int b = 0; b < 6; ++b) {
                    w[2 * b] = philox_u64((uint32_t)c, (uint32_t)q, P | (3u << 4), (uint32_t)b, o->k0, o->k1, 0);
                    w[2 * b + 1] = philox_u64((uint32_t)c, (uint32_t)q, P | (3u << 4), (uint32_t)b, o->k0, o->k1, 1);
                }
                double* vv[3] = {&nvx[to], &nvy[to], &nvz[to]};
                for (int k = 0; k < 3; ++k) {
                    const double th = 2 * M_PI * w[2 * k + 1];
                    *vv[k] = sqrt(r[4]) * sqrt(-log(w[2 * k])) * sin(th) + r[1 + k];
                }
                nir[to] = -log(w[6]) * 0.5 * r[5];
                double x[3];
                place_in_cell(o, c, w[7], w[8], w[9], w[10], w[11], x);
                nx[to] = x[0]; ny[to] = x[1]; nz[to] = x[2];
                continue;
            }
            const int64_t from = sA + perm[q];
            nvx[to] = o->vx[from]; nvy[to] = o->vy[from]; nvz[to] = o->vz[from]; nir[to] = o->ir[from];
            if (q < n0) {
                nx[to] = o->px[from]; ny[to] = o->py[from]; nz[to] = o->pz[from];
            } else {   /* randomlocation of copy j = q - n0 */
                const uint32_t j = (uint32_t)(q - n0);
                double w[6];
                for (int b = 0; b < 3; ++b) {
                    w[2 * b] = philox_u64((uint32_t)c, j, P | (2u << 4), (uint32_t)b, o->k0, o->k1, 0);
                    w[2 * b + 1] = philox_u64((uint32_t)c, j, P | (2u << 4), (uint32_t)b, o->k0, o->k1, 1);
                }
                double x[3];
                place_in_cell(o, c, w[1], w[2], w[3], w[4], w[5], x);
                nx[to] = x[0]; ny[to] = x[1]; nz[to] = x[2];
            }
        }
        if (!upd[c] || n1 == 0) continue;
        /* the linear map, src/ProcessGSIS.cpp:2290-2343 */
        double n = 0.0, u[3] = {0.0, 0.0, 0.0}, T = 0.0, Tr = 0.0;
        for (int q = sB; q < sB + n1; ++q) {
            n += 1.0;
            u[0] += nvx[q]; u[1] += nvy[q]; u[2] += nvz[q];
            T += (nvx[q] * nvx[q] + nvy[q] * nvy[q] + nvz[q] * nvz[q]);
            Tr += nir[q];
        }
        const double Np = n;
        u[0] = u[0] / Np; u[1] = u[1] / Np; u[2] = u[2] / Np;
        const double u2 = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        T = 2.0 / (3.0 * Np) * (T - Np * u2);
        Tr = 4.0 / o->m.dr / Np * Tr;
        double k = 1.0, kr = 1.0, b[3] = {0.0, 0.0, 0.0};
        if (T > 0 && r[4] > 0 && Tr > 0) {
            k = sqrt(r[4] / T);
            b[0] = r[1] - k * u[0]; b[1] = r[2] - k * u[1]; b[2] = r[3] - k * u[2];
            kr = r[5] / Tr;
        }
        for (int q = sB; q < sB + n1; ++q) {
            nvx[q] = k * nvx[q] + b[0];
            nvy[q] = k * nvy[q] + b[1];
            nvz[q] = k * nvz[q] + b[2];
            nir[q] = kr * nir[q];
        }
    }
    free(perm);
    if (!reserve(o, total + 16)) return -3;
    memcpy(o->px, nx, sizeof(double) * (size_t)total); memcpy(o->py, ny, sizeof(double) * (size_t)total);
    memcpy(o->pz, nz, sizeof(double) * (size_t)total); memcpy(o->vx, nvx, sizeof(double) * (size_t)total);
    memcpy(o->vy, nvy, sizeof(double) * (size_t)total); memcpy(o->vz, nvz, sizeof(double) * (size_t)total);
    memcpy(o->ir, nir, sizeof(double) * (size_t)total); memcpy(o->pc, npc, sizeof(int) * (size_t)total);
    memcpy(o->start, nstart, sizeof(int) * ((size_t)ncell + 1));
    free(nx); free(ny); free(nz); free(nvx); free(nvy); free(nvz); free(nir); free(npc); free(nstart);
    free(target); free(upd);
    o->n = total;
    o->nInj = 0;
    o->sorted = 1;
    ++o->gsisEpoch;
    if (report) {
        report[0] = firstNan < ncell ? firstNan : -1;
        report[1] = updated; report[2] = skipped; report[3] = added; report[4] = removed; report[5] = total;
    }
    return 0;
}
