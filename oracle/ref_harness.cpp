/*
 * ref_harness: drives the reference's own DSMC objects (ProcessDSMC,
 * MeshparticalInitial, meshImport from src/) as one compute rank, for the
 * oracle. ORACLE TEST INFRASTRUCTURE: built into oracle/_ref/ from the
 * reference sources where they lie, executed only by tests, the fixture
 * generator and bench.py's reference arm; never part of the product.
 *
 * No reference source is copied or patched. Case constants the reference
 * hard-codes (L0, T_in, T_w in meshImport::setMeshMessage, src/meshImport.cpp:
 * 1316-1318) are handled by overwriting the public `mess` member with a
 * meshMessage image written by the caller; boundary roles by
 * BoundaryConditionTable::addOrReplace (src/BoundaryCondition.h:120-130); the
 * particle RNG by seeding the reference's own thread_rng() generator
 * (src/MeshparticalInitial.h:194-198), which is an inline function-local
 * static shared with the reference translation units.
 *
 * Commands (all files are raw little-endian binaries):
 *   mesh  CAS OUTDIR Ma Kn
 *       readCAS + preprocess (one part) + setMa_Kn_CFL + setMeshMessage +
 *       rootCaptureGlobalDsmcAndReleaseMesh; writes cells.bin, edges.bin,
 *       points.bin, split.bin, mess.bin.
 *   trace CAS MESS PARTS OUT STOPWALL
 *       For every particle, the tracing loop of
 *       ParticleTransportOps::traceParticleDtleft (src/ProcessDSMC.cpp:149-221)
 *       over the public check_intersection2 / CrossboundarySwitch, with the
 *       particle's own dt in dt_left. With STOPWALL=1 the loop stops at the
 *       first wall hit (position advanced to the hit) instead of re-emitting.
 *   advect CAS MESS PARTS OUT ISTEP ROLES
 *       Fills the buckets, runs the public advection(istep) + cache2chain()
 *       and dumps every bucket in bucket order.
 *   run CAS MESS PARTS OUT NSTEPS SEED ROLES AVG_FROM
 *       Runs the reference step loop of src/meshImportTest.cpp:207-234
 *       (preprocesseffquad, advection, cache2chain, collisionDSMC,
 *       statistic_macro) and dumps per-step counters, time-averaged per-cell
 *       step moments, local/record/final_record, crmax, remainders and the
 *       final particles. Prints wall time of the step loop.
 *   gsis CAS MESS PARTS NS ACCEPTED OUT SEED ROLES
 *       Fills the buckets, builds a ProcessGSIS over the rig (no NS solver),
 *       sets its nsresult from NS ([ncell][6] doubles) and, unless ACCEPTED
 *       is "-", its acceptance gate from ACCEPTED ([ncell] bytes), runs the
 *       public molecular_velocity_change() and dumps every bucket.
 *   fill CAS MESS COUNTS OUT SEED
 *       For every cell c with COUNTS[c] > 0 ([ncell] int32), the public
 *       Np_tri_inititial + meshfillpar of MeshparticalInitial (the initial
 *       fill of one cell); dumps every bucket to OUT/particles.bin and the
 *       per-tetrahedron counts, cell after cell, to OUT/np_tri.bin (int32).
 *   fluent CAS MESS FIELDS OUT
 *       readCAS + preprocess, then the public meshImport::out2Fluent_dsmc on
 *       FIELDS ([ncell][18] doubles) with MESS as the case constants, into
 *       OUT/fields.dat; the zone declarations (zonemap: id, first, last) go
 *       to OUT/zones.bin (int32).
 *   sample CAS MESS PARTS OUT NSTEPS PPC [HOSTRULE]
 *       statistic_macroPre, then for every step k = 1..NSTEPS the buckets
 *       are refilled with the step's particles (sampledAt: PARTS thinned
 *       and scaled by a rule of k, PPC particles per cell in PARTS) and the
 *       public statistic_macro(k) runs; with HOSTRULE = 1 the sparse states
 *       are then changed by hostRule after every exchange step, as the GSIS
 *       exchange does. Dumps local, record, final_record, the window
 *       samples and validity and the sparse states.
 *   collide CAS MESS PARTS OUT SEED
 *       Fills the buckets and runs the public collisionDSMC() once from the
 *       initial crmax and remainders (Collision_constant_initial); dumps
 *       the remainders, crmax, the candidate pairs and collisions
 *       (tol_collision_pairs / tol_collision_times, two doubles) and every
 *       bucket.
 *   inject CAS MESS OUT NSTEPS SEED
 *       With no particles in the domain, the public preprocesseffquad(k)
 *       for k = 1..NSTEPS; after each step the injected particles that
 *       stayed in the domain (recv_cache) are collected and the cache is
 *       cleared. Dumps them (OUT/particles.bin), their count per step and
 *       the inflow remainders.
 *   bench CAS MESS COUNTS NSTEPS SEED ROLES UX UY UZ TN
 *       The reference's initial fill as in "fill" (COUNTS[c] particles in
 *       cell c), moved to the freestream the benchmark starts from (the
 *       fill's unit Maxwellian at rest scaled to temperature TN and shifted
 *       by the drift U: v <- U + sqrt(TN) v, Ir <- TN Ir), then ProcessDSMC
 *       over it and NSTEPS steps of the reference's loop (as "run"), each
 *       timed on its own. Prints one JSON line: particles after the fill,
 *       fill seconds, per-step seconds and particles, particle-steps/s.
 *   ROLES is "-" or a comma list tag:role with role in
 *       none,interface,inlet,outlet,wall.
 */
#include "ProcessDSMC.h"
#include "ProcessGSIS.h"
#include "MeshparticalInitial.h"
#include "MessagePassing.h"
#include "meshImport.h"

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

static_assert(sizeof(DsmcCell) == 120, "DsmcCell layout");
static_assert(sizeof(DsmcEdge) == 88, "DsmcEdge layout");
static_assert(sizeof(meshMessage) == 344, "meshMessage layout");

namespace {

struct Particles {
    std::vector<double> px, py, pz, vx, vy, vz, ir, dt;
    std::vector<int> cell;
    std::size_t size() const { return cell.size(); }
};

bool readFile(const std::string& path, std::vector<char>& buf)
{
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) return false;
    std::fseek(f, 0, SEEK_END);
    const long n = std::ftell(f);
    std::fseek(f, 0, SEEK_SET);
    buf.resize((std::size_t)n);
    const bool ok = n == 0 || std::fread(buf.data(), 1, (std::size_t)n, f) == (std::size_t)n;
    std::fclose(f);
    return ok;
}

bool writeFile(const std::string& path, const void* data, std::size_t n)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = n == 0 || std::fwrite(data, 1, n, f) == n;
    std::fclose(f);
    return ok;
}

// particles file: int64 n; 8 double arrays (px,py,pz,vx,vy,vz,Ir,dt); int32 cell[n]
bool readParticles(const std::string& path, Particles& P)
{
    std::vector<char> b;
    if (!readFile(path, b) || b.size() < 8) return false;
    long long n = 0;
    std::memcpy(&n, b.data(), 8);
    const std::size_t need = 8 + (std::size_t)n * (8 * 8 + 4);
    if (b.size() != need) return false;
    std::vector<double>* arr[8] = {&P.px, &P.py, &P.pz, &P.vx, &P.vy, &P.vz, &P.ir, &P.dt};
    const char* p = b.data() + 8;
    for (auto* a : arr) {
        a->resize((std::size_t)n);
        std::memcpy(a->data(), p, (std::size_t)n * 8);
        p += (std::size_t)n * 8;
    }
    P.cell.resize((std::size_t)n);
    std::memcpy(P.cell.data(), p, (std::size_t)n * 4);
    return true;
}

bool writeParticles(const std::string& path, const Particles& P)
{
    std::vector<char> b(8 + P.size() * (8 * 8 + 4));
    long long n = (long long)P.size();
    std::memcpy(b.data(), &n, 8);
    const std::vector<double>* arr[8] = {&P.px, &P.py, &P.pz, &P.vx, &P.vy, &P.vz, &P.ir, &P.dt};
    char* p = b.data() + 8;
    for (auto* a : arr) {
        std::memcpy(p, a->data(), P.size() * 8);
        p += P.size() * 8;
    }
    std::memcpy(p, P.cell.data(), P.size() * 4);
    return writeFile(path, b.data(), b.size());
}

meshImport* loadMesh(const char* cas, double Ma, double Kn)
{
    meshImport* mesh = new meshImport();
    if (!mesh->readCAS(cas)) return nullptr;
    for (int i = 0; i < mesh->Ncell; ++i) mesh->cells[i].no = 0;
    mesh->preprocess(1);
    mesh->rank = 0;
    mesh->c_size = 1;
    mesh->setMa_Kn_CFL(Ma, Kn, 1e2, 1e3, 5);
    mesh->setMeshMessage();
    mesh->rootCaptureGlobalDsmcAndReleaseMesh();
    return mesh;
}

struct Rig {
    meshImport* mesh = nullptr;
    MessagePassing* mpass = nullptr;
    MeshparticalInitial* partinit = nullptr;
    ProcessDSMC* process = nullptr;
    MpiContext ctx;
};

BoundaryRole roleFromName(const std::string& s)
{
    if (s == "interface") return BoundaryRole::Interface;
    if (s == "inlet") return BoundaryRole::Inlet;
    if (s == "outlet") return BoundaryRole::Outlet;
    if (s == "wall") return BoundaryRole::Wall;
    return BoundaryRole::None;
}

void applyRoles(ProcessDSMC& p, const std::string& roles)
{
    if (roles.empty() || roles == "-") return;
    std::size_t pos = 0;
    while (pos < roles.size()) {
        std::size_t comma = roles.find(',', pos);
        if (comma == std::string::npos) comma = roles.size();
        const std::string item = roles.substr(pos, comma - pos);
        const std::size_t colon = item.find(':');
        if (colon != std::string::npos) {
            const int tag = std::atoi(item.substr(0, colon).c_str());
            BoundaryCondition bc = p.boundaryTable.byTag(tag);
            bc.tag = tag;
            bc.dsmcRole = roleFromName(item.substr(colon + 1));
            if (bc.dsmcRole == BoundaryRole::Wall) bc.dsmcModel = BoundaryModel::DiffuseWall;
            if (bc.dsmcRole != BoundaryRole::Inlet) bc.injectParticles = false;
            p.boundaryTable.addOrReplace(bc);
        }
        pos = comma + 1;
    }
    // Interface faces keep their role (the face-cross cache built by the
    // constructor stays valid); boundary lists and emit patches are rebuilt.
    p.rebuildBoundaryDerivedState();
}

// withProcess = false stops before ProcessDSMC, whose constructor takes the
// mesh arrays over from MeshparticalInitial (src/ProcessDSMC.cpp:359-395):
// the reference's own initial fill runs on MeshparticalInitial before that.
bool buildRig(Rig& r, const char* cas, const char* messPath, const std::string& roles, bool withProcess = true)
{
    std::vector<char> mb;
    if (!readFile(messPath, mb) || mb.size() != sizeof(meshMessage)) {
        std::fprintf(stderr, "bad mess file %s\n", messPath);
        return false;
    }
    meshMessage mess;
    std::memcpy(&mess, mb.data(), sizeof(mess));
    r.mesh = loadMesh(cas, mess.Ma, mess.Kn);
    if (!r.mesh) return false;
    r.mesh->mess = mess;
    r.ctx = MpiContext(MPI_COMM_WORLD, MPI_COMM_WORLD);
    r.mpass = new MessagePassing();
    MeshparticalInitial* pi = new MeshparticalInitial();
    const int ncell = r.mesh->Ncell;
    const int nface = r.mesh->Nface;
    pi->mpi = &r.ctx;
    pi->mesh = r.mesh;
    pi->mess = mess;
    pi->mpass = r.mpass;
    pi->comm = r.ctx.comm;
    pi->calGroup = r.ctx.calGroup;
    pi->rank = 0; pi->size = 1; pi->c_rank = 0; pi->c_size = 1;
    pi->cells = r.mesh->Dsmccells;
    pi->edges = r.mesh->Dsmcedges;
    pi->localPointXY = r.mesh->localPointXY;
    pi->faceSplitTag = r.mesh->DsmcfaceSplitTag;
    pi->my_ncell = ncell;
    pi->my_nface = nface;
    pi->my_owned_ncell = ncell;
    pi->local_cells.resize((std::size_t)ncell);
    pi->face_gids.resize((std::size_t)nface);
    for (int i = 0; i < ncell; ++i) { pi->local_cells[(std::size_t)i] = i; pi->gid2local[i] = i; }
    for (int f = 0; f < nface; ++f) { pi->face_gids[(std::size_t)f] = f; pi->face_gid2local[f] = f; }
    pi->rank_cell_all.assign((std::size_t)ncell, 0);
    pi->partitionState.assign(pi->rank_cell_all, 1, 1);
    pi->partitionReady = true;
    pi->cell_particles_curr.assign((std::size_t)ncell, ParticleBucketSoA());
    pi->cell_particle_reserve_hint.assign((std::size_t)ncell, 0);
    pi->Collision_constant_initial();
    r.partinit = pi;
    if (!withProcess) return true;
    r.process = new ProcessDSMC(r.mesh, mess, pi, r.ctx);
    applyRoles(*r.process, roles);
    return true;
}

void fillBuckets(Rig& r, const Particles& P)
{
    for (std::size_t i = 0; i < P.size(); ++i) {
        const int c = P.cell[i];
        ParticleBucketSoA& b = r.partinit->cell_particles_curr[(std::size_t)c];
        particle q;
        q.p_serial = (int)b.size();
        q.p_rank_serial = 0;
        q.p_mesh_serial = c;
        q.p_velocity[0] = P.vx[i]; q.p_velocity[1] = P.vy[i]; q.p_velocity[2] = P.vz[i];
        q.p_location[0] = P.px[i]; q.p_location[1] = P.py[i]; q.p_location[2] = P.pz[i];
        q.p_Ir = P.ir[i];
        q.dt_left = 0.0;
        b.push_back(q);
    }
}

Particles dumpBuckets(Rig& r)
{
    Particles P;
    for (std::size_t c = 0; c < r.partinit->cell_particles_curr.size(); ++c) {
        const ParticleBucketSoA& b = r.partinit->cell_particles_curr[c];
        for (std::size_t i = 0; i < b.size(); ++i) {
            P.px.push_back(b.px[i]); P.py.push_back(b.py[i]); P.pz.push_back(b.pz[i]);
            P.vx.push_back(b.vx[i]); P.vy.push_back(b.vy[i]); P.vz.push_back(b.vz[i]);
            P.ir.push_back(b.p_Ir[i]); P.dt.push_back(b.dt_left[i]);
            P.cell.push_back((int)c);
        }
    }
    return P;
}

int cmdMesh(int argc, char** argv)
{
    if (argc < 6) return 2;
    meshImport* mesh = loadMesh(argv[2], std::atof(argv[4]), std::atof(argv[5]));
    if (!mesh) return 1;
    const std::string out = argv[3];
    bool ok = writeFile(out + "/cells.bin", mesh->Dsmccells.data(), mesh->Dsmccells.size() * sizeof(DsmcCell));
    ok = ok && writeFile(out + "/edges.bin", mesh->Dsmcedges.data(), mesh->Dsmcedges.size() * sizeof(DsmcEdge));
    ok = ok && writeFile(out + "/points.bin", mesh->localPointXY.data(), mesh->localPointXY.size() * sizeof(double));
    ok = ok && writeFile(out + "/split.bin", mesh->DsmcfaceSplitTag.data(), mesh->DsmcfaceSplitTag.size());
    ok = ok && writeFile(out + "/mess.bin", &mesh->mess, sizeof(meshMessage));
    return ok ? 0 : 1;
}

// Trace outputs: per particle
//   int32 cell, ifout, hitFace, hitTri, ncross; double x,y,z, vx,vy,vz, dtleft
int cmdTrace(int argc, char** argv)
{
    if (argc < 7) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], "-")) return 1;
    Particles P;
    if (!readParticles(argv[4], P)) return 1;
    const bool stopWall = std::atoi(argv[6]) != 0;
    const std::size_t n = P.size();
    std::vector<int> ocell(n), oifout(n), oface(n), otri(n), oncross(n);
    std::vector<double> ox(n), oy(n), oz(n), ovx(n), ovy(n), ovz(n), odt(n);
    ProcessDSMC& self = *r.process;
    for (std::size_t i = 0; i < n; ++i) {
        particle part;
        part.p_serial = 0; part.p_rank_serial = 0; part.p_mesh_serial = P.cell[i];
        part.p_location[0] = P.px[i]; part.p_location[1] = P.py[i]; part.p_location[2] = P.pz[i];
        part.p_velocity[0] = P.vx[i]; part.p_velocity[1] = P.vy[i]; part.p_velocity[2] = P.vz[i];
        part.p_Ir = P.ir[i]; part.dt_left = 0.0;
        int cellid = P.cell[i];
        int crossfid = -1;
        int tag = -1;
        double dtleft = P.dt[i];
        int ifout = 0;
        int hitFace = -1, hitTri = 0, ncross = 0;
        double t = 0.0;
        // loop of traceParticleDtleft, src/ProcessDSMC.cpp:155-219 (inclusive_hit = true)
        while (dtleft > 0.0) {
            crossfid = self.check_intersection2(&part, cellid, t, crossfid, tag);
            if (crossfid == -2 || !std::isfinite(t) || t <= 0.0) { ifout = -1; dtleft = 0.0; break; }
            if (t >= dtleft) { self.scalar_product(part.p_location, part.p_velocity, dtleft, DIM); dtleft = 0.0; break; }
            const BoundaryRole role = self.boundaryTable.byTag(self.edges[(std::size_t)crossfid].faceTag).dsmcRole;
            if (role != BoundaryRole::Interface && hitFace < 0) {
                hitFace = crossfid; hitTri = tag;
                if (stopWall && role == BoundaryRole::Wall) {
                    self.scalar_product(part.p_location, part.p_velocity, t, DIM);
                    dtleft -= t;
                    break;
                }
            }
            ++ncross;
            self.CrossboundarySwitch(&part, cellid, ifout, dtleft, crossfid, t, tag);
            if (ifout == -1 || cellid == -1) { dtleft = 0.0; break; }
        }
        ocell[i] = cellid; oifout[i] = ifout; oface[i] = hitFace; otri[i] = hitTri; oncross[i] = ncross;
        ox[i] = part.p_location[0]; oy[i] = part.p_location[1]; oz[i] = part.p_location[2];
        ovx[i] = part.p_velocity[0]; ovy[i] = part.p_velocity[1]; ovz[i] = part.p_velocity[2];
        odt[i] = dtleft;
    }
    FILE* f = std::fopen(argv[5], "wb");
    if (!f) return 1;
    long long nn = (long long)n;
    std::fwrite(&nn, 8, 1, f);
    for (auto* a : {&ocell, &oifout, &oface, &otri, &oncross}) std::fwrite(a->data(), 4, n, f);
    for (auto* a : {&ox, &oy, &oz, &ovx, &ovy, &ovz, &odt}) std::fwrite(a->data(), 8, n, f);
    std::fclose(f);
    return 0;
}

int cmdAdvect(int argc, char** argv)
{
    if (argc < 8) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], argv[7])) return 1;
    Particles P;
    if (!readParticles(argv[4], P)) return 1;
    fillBuckets(r, P);
    const int istep = std::atoi(argv[6]);
    r.process->advection(istep);
    r.process->cache2chain();
    return writeParticles(argv[5], dumpBuckets(r)) ? 0 : 1;
}

int cmdRun(int argc, char** argv)
{
    if (argc < 10) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], argv[8])) return 1;
    Particles P;
    if (!readParticles(argv[4], P)) return 1;
    const std::string out = argv[5];
    const int nsteps = std::atoi(argv[6]);
    const unsigned seed = (unsigned)std::strtoul(argv[7], nullptr, 10);
    const int avgFrom = std::atoi(argv[9]);
    r.partinit->thread_rng().seed(seed);
    std::srand(seed);
    fillBuckets(r, P);
    ProcessDSMC& p = *r.process;
    const int ncell = p.iNcell;
    p.statistic_macroPre();
    std::vector<double> avg((std::size_t)ncell * 18, 0.0);
    std::vector<long long> perStep((std::size_t)nsteps * 4, 0);
    double tStep = 0.0;
    long long particleSteps = 0;
    for (int istep = 1; istep <= nsteps; ++istep) {
        long long nBefore = 0;
        for (const auto& b : r.partinit->cell_particles_curr) nBefore += (long long)b.size();
        const auto t0 = std::chrono::steady_clock::now();
        p.preprocesseffquad(istep);
        const long long injected = (long long)p.recv_cache.size();
        p.advection(istep);
        p.cache2chain();
        p.collisionDSMC();
        p.statistic_macro(istep);
        tStep += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        particleSteps += nBefore;
        long long nAfter = 0;
        for (const auto& b : r.partinit->cell_particles_curr) nAfter += (long long)b.size();
        perStep[(std::size_t)(istep - 1) * 4 + 0] = nAfter;
        perStep[(std::size_t)(istep - 1) * 4 + 1] = injected;
        perStep[(std::size_t)(istep - 1) * 4 + 2] = p.tol_collision_pairs;
        perStep[(std::size_t)(istep - 1) * 4 + 3] = p.tol_collision_times;
        if (istep >= avgFrom) {
            for (int c = 0; c < ncell; ++c) {
                double* a = &avg[(std::size_t)c * 18];
                a[0] += p.step_rho[(std::size_t)c];
                for (int k = 0; k < 3; ++k) a[1 + k] += p.step_U[(std::size_t)c * 3 + k];
                a[4] += p.step_T[(std::size_t)c];
                for (int k = 0; k < 6; ++k) a[5 + k] += p.step_sigma[(std::size_t)c * 6 + k];
                for (int k = 0; k < 3; ++k) a[11 + k] += p.step_q[(std::size_t)c * 3 + k];
                for (int k = 0; k < 4; ++k) a[14 + k] += p.step_qr[(std::size_t)c * 4 + k];
            }
        }
    }
    bool ok = writeFile(out + "/steps.bin", perStep.data(), perStep.size() * 8);
    ok = ok && writeFile(out + "/moments.bin", avg.data(), avg.size() * 8);
    ok = ok && writeFile(out + "/local.bin", p.local.data(), p.local.size() * 8);
    ok = ok && writeFile(out + "/record.bin", p.record.data(), p.record.size() * 8);
    ok = ok && writeFile(out + "/final_record.bin", p.final_record.data(), p.final_record.size() * 8);
    ok = ok && writeFile(out + "/crmax.bin", r.partinit->crmax.data(), r.partinit->crmax.size() * 8);
    ok = ok && writeFile(out + "/remcoll.bin", r.partinit->remainderincoll.data(), r.partinit->remainderincoll.size() * 8);
    ok = ok && writeFile(out + "/reminj.bin", r.partinit->remainderinpre.data(), r.partinit->remainderinpre.size() * 8);
    ok = ok && writeFile(out + "/window_samples.bin", p.dsmc2ns_window_samples.data(), p.dsmc2ns_window_samples.size() * 8);
    ok = ok && writeFile(out + "/sparse_state.bin", p.dsmc2ns_sparse_state.data(), p.dsmc2ns_sparse_state.size());
    ok = ok && writeParticles(out + "/particles.bin", dumpBuckets(r));
    std::printf("{\"steps\": %d, \"particle_steps\": %lld, \"seconds\": %.6f, \"particle_steps_per_s\": %.3f}\n",
                nsteps, particleSteps, tStep, tStep > 0 ? (double)particleSteps / tStep : 0.0);
    return ok ? 0 : 1;
}

int cmdGsis(int argc, char** argv)
{
    if (argc < 10) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], argv[9])) return 1;
    Particles P;
    if (!readParticles(argv[4], P)) return 1;
    const int ncell = r.process->iNcell;
    std::vector<char> nsb;
    if (!readFile(argv[5], nsb) || nsb.size() != (std::size_t)ncell * 6 * 8) {
        std::fprintf(stderr, "bad NS file %s\n", argv[5]);
        return 1;
    }
    const unsigned seed = (unsigned)std::strtoul(argv[8], nullptr, 10);
    r.partinit->thread_rng().seed(seed);
    std::srand(seed);
    fillBuckets(r, P);
    ProcessGSIS g(r.mesh, r.process, r.partinit, nullptr, r.ctx);
    g.nsresult.resize((std::size_t)ncell * 6);
    std::memcpy(g.nsresult.data(), nsb.data(), nsb.size());
    const std::string acc = argv[6];
    if (acc != "-") {
        std::vector<char> ab;
        if (!readFile(acc, ab) || ab.size() != (std::size_t)ncell) return 1;
        g.dsmc2ns_macro_accepted.assign(ab.begin(), ab.end());
        g.dsmc2ns_acceptance_ready = true;
    }
    g.molecular_velocity_change();
    return writeParticles(argv[7], dumpBuckets(r)) ? 0 : 1;
}

int cmdFill(int argc, char** argv)
{
    if (argc < 7) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], "-", false)) return 1;
    const int ncell = r.partinit->my_ncell;
    std::vector<char> cb;
    if (!readFile(argv[4], cb) || cb.size() != (std::size_t)ncell * 4) return 1;
    const unsigned seed = (unsigned)std::strtoul(argv[6], nullptr, 10);
    r.partinit->thread_rng().seed(seed);
    std::srand(seed);
    const std::string out = argv[5];
    std::vector<int> npTri;
    for (int c = 0; c < ncell; ++c) {
        int np = 0;
        std::memcpy(&np, cb.data() + (std::size_t)c * 4, 4);
        if (np <= 0) continue;
        std::vector<double> tri;
        r.partinit->Np_tri_inititial(c, tri, np);
        for (double t : tri) npTri.push_back((int)t);
        if (!tri.empty()) r.partinit->meshfillpar(c, tri);
    }
    bool ok = writeParticles(out + "/particles.bin", dumpBuckets(r));
    return ok && writeFile(out + "/np_tri.bin", npTri.data(), npTri.size() * 4) ? 0 : 1;
}

int cmdBench(int argc, char** argv)
{
    if (argc < 12) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], "-", false)) return 1;
    const int ncell = r.partinit->my_ncell;
    std::vector<char> cb;
    if (!readFile(argv[4], cb) || cb.size() != (std::size_t)ncell * 4) return 1;
    const int nsteps = std::atoi(argv[5]);
    const unsigned seed = (unsigned)std::strtoul(argv[6], nullptr, 10);
    const std::string roles = argv[7];
    const double u[3] = {std::atof(argv[8]), std::atof(argv[9]), std::atof(argv[10])};
    const double tN = std::atof(argv[11]);
    const double sq = std::sqrt(tN);
    r.partinit->thread_rng().seed(seed);
    std::srand(seed);
    const auto f0 = std::chrono::steady_clock::now();
    for (int c = 0; c < ncell; ++c) {
        int np = 0;
        std::memcpy(&np, cb.data() + (std::size_t)c * 4, 4);
        if (np <= 0) continue;
        std::vector<double> tri;
        r.partinit->Np_tri_inititial(c, tri, np);
        if (!tri.empty()) r.partinit->meshfillpar(c, tri);
    }
    long long n0 = 0;
    for (auto& b : r.partinit->cell_particles_curr) {
        for (std::size_t i = 0; i < b.size(); ++i) {
            b.vx[i] = u[0] + sq * b.vx[i];
            b.vy[i] = u[1] + sq * b.vy[i];
            b.vz[i] = u[2] + sq * b.vz[i];
            b.p_Ir[i] = tN * b.p_Ir[i];
        }
        n0 += (long long)b.size();
    }
    const double fillSeconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - f0).count();
    r.process = new ProcessDSMC(r.mesh, r.mesh->mess, r.partinit, r.ctx);
    applyRoles(*r.process, roles);
    ProcessDSMC& p = *r.process;
    p.statistic_macroPre();
    std::vector<double> sec((std::size_t)nsteps);
    std::vector<long long> parts((std::size_t)nsteps);
    double total = 0.0;
    long long particleSteps = 0;
    for (int istep = 1; istep <= nsteps; ++istep) {
        long long nBefore = 0;
        for (const auto& b : r.partinit->cell_particles_curr) nBefore += (long long)b.size();
        const auto t0 = std::chrono::steady_clock::now();
        p.preprocesseffquad(istep);
        p.advection(istep);
        p.cache2chain();
        p.collisionDSMC();
        p.statistic_macro(istep);
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        sec[(std::size_t)istep - 1] = dt;
        parts[(std::size_t)istep - 1] = nBefore;
        total += dt;
        particleSteps += nBefore;
    }
    std::printf("{\"particles\": %lld, \"fill_seconds\": %.6f, \"steps\": %d, \"particle_steps\": %lld, "
                "\"seconds\": %.6f, \"particle_steps_per_s\": %.3f, \"step_seconds\": [",
                n0, fillSeconds, nsteps, particleSteps, total, total > 0 ? (double)particleSteps / total : 0.0);
    for (int k = 0; k < nsteps; ++k) std::printf("%s%.6f", k ? ", " : "", sec[(std::size_t)k]);
    std::printf("], \"step_particles\": [");
    for (int k = 0; k < nsteps; ++k) std::printf("%s%lld", k ? ", " : "", parts[(std::size_t)k]);
    std::printf("]}\n");
    return 0;
}

// The particles sampled at step k in the "sample" command: particle i of
// the input (cell c) is present unless c % 5 == 0 and (k % 50 != 0 or
// i % PPC != 0) (such cells hold one particle on two steps of every
// 100: sparse windows), or c % 5 == 1 and (k + i) % 3 == 0; velocities are
// scaled by s = 1 + (k % 8) / 16 and Ir by s * s (both exact in binary).
bool sampledAt(int k, std::size_t i, int c, int ppc)
{
    if (c % 5 == 0) return k % 50 == 0 && (int)(i % (std::size_t)ppc) == 0;
    if (c % 5 == 1) return (k + (long long)i) % 3 != 0;
    return true;
}

// The host rule of the "sample" command (HOSTRULE = 1), standing in for the
// sparse-state decisions of ProcessGSIS::DSMC2NS (src/ProcessGSIS.cpp:
// 1660-1674) after exchange step k (k % 100 == 0), j = k / 100: a normal
// cell c with c % 7 == 3 becomes accumulating when j is odd; an
// accumulating cell with c % 3 == 0 is released when j is even.
unsigned char hostRule(unsigned char st, int c, int k)
{
    const int j = k / 100;
    if (st == ProcessDSMC::DSMC2NS_SPARSE_NORMAL && c % 7 == 3 && j % 2 == 1)
        return ProcessDSMC::DSMC2NS_SPARSE_ACCUMULATING;
    if (st == ProcessDSMC::DSMC2NS_SPARSE_ACCUMULATING && c % 3 == 0 && j % 2 == 0)
        return ProcessDSMC::DSMC2NS_SPARSE_RELEASED;
    return st;
}

int cmdSample(int argc, char** argv)
{
    if (argc < 8) return 2;
    const bool rule = argc > 8 && std::atoi(argv[8]) != 0;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], "-")) return 1;
    Particles P;
    if (!readParticles(argv[4], P)) return 1;
    const std::string out = argv[5];
    const int nsteps = std::atoi(argv[6]);
    const int ppc = std::atoi(argv[7]);
    ProcessDSMC& p = *r.process;
    p.statistic_macroPre();
    for (int k = 1; k <= nsteps; ++k) {
        for (auto& b : r.partinit->cell_particles_curr) b.clear();
        const double s = 1.0 + (double)(k % 8) / 16.0;
        Particles Q;
        for (std::size_t i = 0; i < P.size(); ++i) {
            if (!sampledAt(k, i, P.cell[i], ppc)) continue;
            Q.px.push_back(P.px[i]); Q.py.push_back(P.py[i]); Q.pz.push_back(P.pz[i]);
            Q.vx.push_back(P.vx[i] * s); Q.vy.push_back(P.vy[i] * s); Q.vz.push_back(P.vz[i] * s);
            Q.ir.push_back(P.ir[i] * (s * s)); Q.dt.push_back(0.0); Q.cell.push_back(P.cell[i]);
        }
        fillBuckets(r, Q);
        p.statistic_macro(k);
        if (rule && k % 100 == 0)
            for (std::size_t c = 0; c < p.dsmc2ns_sparse_state.size(); ++c)
                p.dsmc2ns_sparse_state[c] = hostRule(p.dsmc2ns_sparse_state[c], (int)c, k);
    }
    std::vector<double> wv(p.dsmc2ns_window_valid.begin(), p.dsmc2ns_window_valid.end());
    bool ok = writeFile(out + "/local.bin", p.local.data(), p.local.size() * 8);
    ok = ok && writeFile(out + "/record.bin", p.record.data(), p.record.size() * 8);
    ok = ok && writeFile(out + "/final_record.bin", p.final_record.data(), p.final_record.size() * 8);
    ok = ok && writeFile(out + "/window_samples.bin", p.dsmc2ns_window_samples.data(), p.dsmc2ns_window_samples.size() * 8);
    ok = ok && writeFile(out + "/window_valid.bin", wv.data(), wv.size() * 8);
    ok = ok && writeFile(out + "/sparse_state.bin", p.dsmc2ns_sparse_state.data(), p.dsmc2ns_sparse_state.size());
    return ok ? 0 : 1;
}

int cmdCollide(int argc, char** argv)
{
    if (argc < 7) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], "-")) return 1;
    Particles P;
    if (!readParticles(argv[4], P)) return 1;
    const std::string out = argv[5];
    const unsigned seed = (unsigned)std::strtoul(argv[6], nullptr, 10);
    r.partinit->thread_rng().seed(seed);
    std::srand(seed);
    fillBuckets(r, P);
    ProcessDSMC& p = *r.process;
    p.collisionDSMC();
    const double counts[2] = {(double)p.tol_collision_pairs, (double)p.tol_collision_times};
    bool ok = writeFile(out + "/remcoll.bin", r.partinit->remainderincoll.data(), r.partinit->remainderincoll.size() * 8);
    ok = ok && writeFile(out + "/crmax.bin", r.partinit->crmax.data(), r.partinit->crmax.size() * 8);
    ok = ok && writeFile(out + "/counts.bin", counts, sizeof counts);
    ok = ok && writeParticles(out + "/particles.bin", dumpBuckets(r));
    return ok ? 0 : 1;
}

int cmdInject(int argc, char** argv)
{
    if (argc < 6) return 2;
    Rig r;
    if (!buildRig(r, argv[2], argv[3], "-")) return 1;
    const std::string out = argv[4];
    const int nsteps = std::atoi(argv[5]);
    const unsigned seed = (unsigned)std::strtoul(argv[6], nullptr, 10);
    r.partinit->thread_rng().seed(seed);
    std::srand(seed);
    ProcessDSMC& p = *r.process;
    Particles Q;
    std::vector<long long> perStep((std::size_t)nsteps, 0);
    for (int k = 1; k <= nsteps; ++k) {
        p.preprocesseffquad(k);
        perStep[(std::size_t)(k - 1)] = (long long)p.recv_cache.size();
        for (const particle& q : p.recv_cache) {
            Q.px.push_back(q.p_location[0]); Q.py.push_back(q.p_location[1]); Q.pz.push_back(q.p_location[2]);
            Q.vx.push_back(q.p_velocity[0]); Q.vy.push_back(q.p_velocity[1]); Q.vz.push_back(q.p_velocity[2]);
            Q.ir.push_back(q.p_Ir); Q.dt.push_back(q.dt_left); Q.cell.push_back(q.p_mesh_serial);
        }
        p.recv_cache.clear();
    }
    bool ok = writeParticles(out + "/particles.bin", Q);
    ok = ok && writeFile(out + "/steps.bin", perStep.data(), perStep.size() * 8);
    ok = ok && writeFile(out + "/reminj.bin", r.partinit->remainderinpre.data(), r.partinit->remainderinpre.size() * 8);
    return ok ? 0 : 1;
}

int cmdFluent(int argc, char** argv)
{
    if (argc < 6) return 2;
    std::vector<char> mb;
    if (!readFile(argv[3], mb) || mb.size() != sizeof(meshMessage)) return 1;
    meshMessage mess;
    std::memcpy(&mess, mb.data(), sizeof(mess));
    meshImport* mesh = loadMesh(argv[2], mess.Ma, mess.Kn);
    if (!mesh) return 1;
    mesh->mess = mess;
    std::vector<char> wb;
    if (!readFile(argv[4], wb) || wb.size() % (18 * 8) != 0) return 1;
    std::vector<double> w(wb.size() / 8);
    std::memcpy(w.data(), wb.data(), wb.size());
    const std::string out = argv[5];
    if (!mesh->out2Fluent_dsmc((out + "/fields.dat").c_str(), w.data())) return 1;
    std::vector<int> z;
    for (const ZONE& zn : mesh->zonemap) {
        z.push_back(zn.id);
        z.push_back(zn.firstidx);
        z.push_back(zn.lastidx);
    }
    return writeFile(out + "/zones.bin", z.data(), z.size() * 4) ? 0 : 1;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 2) {
        std::fprintf(stderr, "usage: ref_harness mesh|trace|advect|run ...\n");
        return 2;
    }
    const std::string cmd = argv[1];
    if (cmd == "mesh") return cmdMesh(argc, argv);
    if (cmd == "trace") return cmdTrace(argc, argv);
    if (cmd == "bench") return cmdBench(argc, argv);
    if (cmd == "advect") return cmdAdvect(argc, argv);
    if (cmd == "run") return cmdRun(argc, argv);
    if (cmd == "gsis") return cmdGsis(argc, argv);
    if (cmd == "fill") return cmdFill(argc, argv);
    if (cmd == "fluent") return cmdFluent(argc, argv);
    if (cmd == "sample") return cmdSample(argc, argv);
    if (cmd == "collide") return cmdCollide(argc, argv);
    if (cmd == "inject") return cmdInject(argc, argv);
    std::fprintf(stderr, "unknown command %s\n", cmd.c_str());
    return 2;
}
