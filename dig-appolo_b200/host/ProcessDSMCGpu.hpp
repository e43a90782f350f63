// ProcessDSMCGpu: the reference's ProcessDSMC interface for the DSMC
// particle step (src/ProcessDSMC.h:441-492), on the B200 library's C-ABI
// (include/dsmc_gpu.h). Header only, C++17; link with -ldsmcgpu.
//
// Same member names and argument meaning as the reference:
//   preprocesseffquad(istep), advection(istep), cache2chain(),
//   collisionDSMC(), statistic_macro(istep), statistic_macroPre(),
//   out2dat(istep), outBoundaryStressHeat(istep)
// and the per-cell fields the host GSIS step reads (local, record,
// final_record, [ncell][18] in MacroIndex order). One object owns one
// device-resident case (all cells of the mesh: one domain).
//
// Errors: the reference prints and aborts (e.g. src/ProcessDSMC.cpp:874);
// here a failed call throws DsmcError carrying the library's message
// (dsmc_last_error), and the object stays usable where the library allows.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "dsmc_gpu.h"
#include "dsmc_meshio.h"

namespace dsmc_b200 {

class DsmcError : public std::runtime_error {
public:
    explicit DsmcError(const std::string& m) : std::runtime_error(m) {}
};

// Particles as structure-of-arrays host vectors (cell_particles_curr
// flattened; src/MeshparticalInitial.h:229).
struct Particles {
    std::vector<double> x, y, z, vx, vy, vz, ir;
    std::vector<int32_t> cell;
    size_t size() const { return cell.size(); }
};

// One wall face of outBoundaryStressHeat's output
// (src/ProcessDSMC.cpp:3498-3550): normal (outward), pressure, shear
// vector, stress vector, translational / rotational / total heat flux,
// normalised by n_ref like the reference's Fluent sections.
struct WallFaceFields {
    int face = -1;
    double normal[3] = {0.0, 0.0, 0.0};
    double pressure = 0.0;
    double shear[3] = {0.0, 0.0, 0.0};
    double stress[3] = {0.0, 0.0, 0.0};
    double qTrans = 0.0, qRot = 0.0, qTotal = 0.0;
};

// A Fluent ASCII case read by the library (meshImport's readCAS +
// preprocess + the DSMC topology, for one partition): the arrays
// ProcessDSMCGpu takes, the zone declarations (zonemap) and the case
// constants (setMeshMessage / setParticleMessage).
class MeshFile {
public:
    explicit MeshFile(const std::string& casPath)
    {
        if (dsmc_mesh_read_cas(casPath.c_str(), &m_) != DSMC_OK) throw DsmcError(dsmc_meshio_last_error());
    }
    ~MeshFile() { dsmc_mesh_free(m_); }
    MeshFile(const MeshFile&) = delete;
    MeshFile& operator=(const MeshFile&) = delete;

    DsmcMeshDesc desc() const
    {
        DsmcMeshDesc md{};
        dsmc_mesh_get_desc(m_, &md);
        return md;
    }
    std::vector<DsmcZone> zonemap() const
    {
        int32_t n = 0;
        dsmc_mesh_get_zones(m_, nullptr, 0, &n);
        std::vector<DsmcZone> z((size_t)n);
        dsmc_mesh_get_zones(m_, z.data(), n, &n);
        return z;
    }
    // the reference's constants: L0 3.912, T_in 142.2, T_wall 300, 100 per cell
    DsmcMeshMessage message(double Ma, double Kn, int ppc = 100, double L0 = 3.912, double T_in = 142.2,
                            double T_wall = 300.0, double cfl = 1e2, double cfl_ns = 5.0) const
    {
        DsmcMeshMessage mm{};
        if (dsmc_mesh_message(m_, Ma, Kn, ppc, L0, T_in, T_wall, cfl, cfl_ns, &mm) != DSMC_OK)
            throw DsmcError(dsmc_meshio_last_error());
        return mm;
    }

private:
    DsmcMeshFile* m_ = nullptr;
};

class ProcessDSMCGpu {
public:
    static constexpr int Madata = DSMC_MACRO_WIDTH;   // MacroIndex count (src/ProcessDSMC.h:28-49)

    // The mesh arrays are the reference's own (DsmcCell, DsmcEdge,
    // localPointXY, faceSplitTag after rootCaptureGlobalDsmcAndReleaseMesh);
    // they are copied at construction.
    ProcessDSMCGpu(const DsmcMeshDesc& mesh, const DsmcMeshMessage& mess, const DsmcCaseParams& params,
                   int device = 0)
        : mess_(mess), params_(params), ncell_(mesh.ncell), nface_(mesh.nface),
          edges_(mesh.edges, mesh.edges + mesh.nface)
    {
        if (dsmc_create(&mesh, &mess, &params, device, &h_) != DSMC_OK)
            throw DsmcError(std::string("dsmc_create: ") + dsmc_last_error(nullptr));
        // zone declarations as a case file makes them: the cell zone 2 and
        // one face zone per run of equal face tags
        zonemap.push_back(DsmcZone{12, 2, 1, ncell_});
        for (int f = 0; f < nface_;) {
            int g = f;
            while (g < nface_ && edges_[(size_t)g].faceTag == edges_[(size_t)f].faceTag) ++g;
            zonemap.push_back(DsmcZone{13, edges_[(size_t)f].faceTag, f + 1, g});
            f = g;
        }
    }
    // From a case file: its arrays and its zone declarations.
    ProcessDSMCGpu(const MeshFile& mesh, const DsmcMeshMessage& mess, const DsmcCaseParams& params, int device = 0)
        : ProcessDSMCGpu(mesh.desc(), mess, params, device)
    {
        zonemap = mesh.zonemap();
    }

    // meshImport::zonemap (src/meshImport.h:120-129): the zones out2dat and
    // outBoundaryStressHeat write
    std::vector<DsmcZone> zonemap;
    ~ProcessDSMCGpu()
    {
        if (h_) dsmc_destroy(h_);
    }
    ProcessDSMCGpu(const ProcessDSMCGpu&) = delete;
    ProcessDSMCGpu& operator=(const ProcessDSMCGpu&) = delete;
    ProcessDSMCGpu(ProcessDSMCGpu&& o) noexcept { *this = std::move(o); }
    ProcessDSMCGpu& operator=(ProcessDSMCGpu&& o) noexcept
    {
        if (this != &o) {
            if (h_) dsmc_destroy(h_);
            h_ = o.h_; o.h_ = nullptr;
            mess_ = o.mess_; params_ = o.params_; ncell_ = o.ncell_; nface_ = o.nface_;
            edges_ = std::move(o.edges_);
            zonemap = std::move(o.zonemap);
        }
        return *this;
    }

    // ---- particles
    void uploadParticles(const Particles& p)
    {
        check(dsmc_upload_particles(h_, (int64_t)p.size(), p.x.data(), p.y.data(), p.z.data(), p.vx.data(),
                                    p.vy.data(), p.vz.data(), p.ir.data(), p.cell.data()),
              "dsmc_upload_particles");
    }
    int64_t particleCount() const
    {
        int64_t n = 0;
        check(dsmc_particle_count(h_, &n), "dsmc_particle_count");
        return n;
    }
    Particles downloadParticles() const
    {
        const int64_t n = particleCount();
        Particles p;
        for (auto* v : {&p.x, &p.y, &p.z, &p.vx, &p.vy, &p.vz, &p.ir}) v->resize((size_t)n);
        p.cell.resize((size_t)n);
        check(dsmc_download_particles(h_, n, p.x.data(), p.y.data(), p.z.data(), p.vx.data(), p.vy.data(),
                                      p.vz.data(), p.ir.data(), p.cell.data(), nullptr),
              "dsmc_download_particles");
        return p;
    }

    // ---- the initial fill on the device: MeshparticalInitial's own
    // (Np_tri_inititial / meshfillpar, src/MeshparticalInitial.cpp:413-418,
    // 481-721: a unit Maxwellian at rest), or the same placement with the
    // case's freestream (the state the coupled start-up's first GSIS update
    // shifts the fill to)
    void initialFill(double ppcMean, uint64_t seed)
    {
        check(dsmc_fill_initial(h_, ppcMean, seed), "dsmc_fill_initial");
    }
    void freestreamFill(double ppcMean, uint64_t seed)
    {
        check(dsmc_fill_freestream(h_, ppcMean, seed), "dsmc_fill_freestream");
    }

    // ---- the reference's step (src/meshImportTest.cpp:207-234)
    void preprocesseffquad(int istep) { check(dsmc_preprocesseffquad(h_, istep), "preprocesseffquad"); }
    void advection(int istep) { check(dsmc_advection(h_, istep), "advection"); }
    void cache2chain() { check(dsmc_cache2chain(h_), "cache2chain"); }
    void collisionDSMC() { check(dsmc_collisionDSMC(h_), "collisionDSMC"); }
    void statistic_macro(int istep) { check(dsmc_statistic_macro(h_, istep), "statistic_macro"); }
    void statistic_macroPre() { check(dsmc_statistic_macroPre(h_), "statistic_macroPre"); }
    // the five calls above as one CUDA-graph replay (same kernels, same bits)
    void step(int istep) { check(dsmc_step(h_, istep, DSMC_STAGE_ALL), "dsmc_step"); }

    // ---- fields for the host GSIS step, [ncell][18] FP64 in MacroIndex order
    std::vector<double> local() const { return macro(DSMC_MACRO_LOCAL); }
    std::vector<double> record() const { return macro(DSMC_MACRO_RECORD); }
    std::vector<double> final_record() const { return macro(DSMC_MACRO_FINAL_RECORD); }
    std::vector<int32_t> particlesPerCell() const
    {
        std::vector<int32_t> ppc((size_t)ncell_);
        check(dsmc_download_counts(h_, ppc.data(), nullptr, nullptr, nullptr, nullptr, nullptr), "counts");
        return ppc;
    }
    std::vector<unsigned char> sparseState() const
    {
        std::vector<unsigned char> st((size_t)ncell_);
        check(dsmc_download_counts(h_, nullptr, nullptr, nullptr, st.data(), nullptr, nullptr), "counts");
        return st;
    }
    // dsmc2ns_sparse_state as ProcessGSIS::DSMC2NS leaves it (1 accumulating,
    // 2 released; src/ProcessGSIS.cpp:1660-1674), written back for the steps
    void setSparseState(const std::vector<unsigned char>& st)
    {
        if ((int)st.size() != ncell_) throw DsmcError("setSparseState: one state per cell");
        check(dsmc_upload_sparse_state(h_, st.data()), "dsmc_upload_sparse_state");
    }

    // The field set out2dat writes (src/ProcessDSMC.cpp:3338-3377): record
    // up to NSS and for sparse cells (states 1, 2), final_record after.
    std::vector<double> out2datFields(int istep) const
    {
        std::vector<double> rec = record();
        if (istep <= params_.nss) return rec;
        const std::vector<double> fin = final_record();
        const std::vector<unsigned char> st = sparseState();
        for (int c = 0; c < ncell_; ++c) {
            if (st[(size_t)c] == 1 || st[(size_t)c] == 2) continue;
            for (int j = 0; j < Madata; ++j) rec[(size_t)c * Madata + j] = fin[(size_t)c * Madata + j];
        }
        return rec;
    }

    // out2dat (src/ProcessDSMC.cpp:3338-3438): the fields of out2datFields
    // as meshImport::out2Fluent_dsmc writes them (Fluent sections 700-712
    // of cell zone 2). The reference's path is
    // ./statisticResults/DSMCKn%.1f_iter%d_CELL%d.dat (defaultOut2datPath).
    bool out2dat(int istep, const std::string& path) const
    {
        check(dsmc_out2dat(h_, istep, zonemap.data(), (int32_t)zonemap.size(), path.c_str()), "dsmc_out2dat");
        return true;
    }
    std::string defaultOut2datPath(int istep) const
    {
        char b[200];
        std::snprintf(b, sizeof b, "./statisticResults/DSMCKn%.1f_iter%d_CELL%d.dat", mess_.Kn, istep, mess_.Ncell);
        return b;
    }

    // outBoundaryStressHeat's conversion (src/ProcessDSMC.cpp:3451-3550):
    // steady wall tallies (hits, momentum and energy deltas, accumulated
    // after NSS) to pressure, shear and heat flux per wall face, scaled by
    // 2 Neff / (dt * steps) / area / n_ref. Only faces whose zone is a
    // diffuse wall are returned.
    std::vector<WallFaceFields> boundaryStressHeat(int istep) const
    {
        std::vector<double> raw((size_t)nface_ * 6);
        check(dsmc_download_wall(h_, raw.data()), "dsmc_download_wall");
        const bool steady = istep > params_.nss;
        const double sampleSteps = steady ? (double)(istep - params_.nss) : 1.0;
        const double timeScale = (mess_.dtime > 0.0 && sampleSteps > 0.0) ? mess_.Neff / (mess_.dtime * sampleSteps) : 0.0;
        std::vector<WallFaceFields> out;
        for (int f = 0; f < nface_; ++f) {
            const DsmcEdgeRec& e = edges_[(size_t)f];
            if (roleOf(e.faceTag) != DSMC_ROLE_WALL) continue;
            WallFaceFields w;
            w.face = f;
            double n[3] = {e.edgeNormal[0], e.edgeNormal[1], e.edgeNormal[2]};
            const double len = std::sqrt(n[0] * n[0] + n[1] * n[1] + n[2] * n[2]);
            if (len > 0.0 && std::isfinite(len)) {
                for (double& v : n) v /= len;
            } else {
                n[0] = 1.0; n[1] = 0.0; n[2] = 0.0;
            }
            const double ni[3] = {-n[0], -n[1], -n[2]};
            const double* in = &raw[(size_t)f * 6];
            const double pn = in[1] * ni[0] + in[2] * ni[1] + in[3] * ni[2];
            const double pt[3] = {in[1] - pn * ni[0], in[2] - pn * ni[1], in[3] - pn * ni[2]};
            const double area = (e.length > 0.0 && std::isfinite(e.length)) ? e.length : 1.0;
            const double scale = (area > 0.0 && mess_.n_ref > 0.0) ? 2.0 * timeScale / area / mess_.n_ref : 0.0;
            for (int d = 0; d < 3; ++d) w.normal[d] = n[d];
            w.pressure = pn * scale;
            for (int d = 0; d < 3; ++d) w.shear[d] = -pt[d] * scale;
            for (int d = 0; d < 3; ++d) w.stress[d] = w.pressure * w.normal[d] + w.shear[d];
            w.qTrans = -in[4] * scale;
            w.qRot = -in[5] * scale;
            w.qTotal = w.qTrans + w.qRot;
            out.push_back(w);
        }
        return out;
    }

    // outBoundaryStressHeat (src/ProcessDSMC.cpp:3451-3652): the fields
    // above as Fluent sections 700-706 of every all-wall zone. Returns true
    // with nothing written when wall statistics are off (the reference's
    // build has them off) or no zone is all wall. The reference's path is
    // ./statisticResults/BoundaryStressHeatFluentKn%.1f_iter%d.dat.
    bool outBoundaryStressHeat(int istep, const std::string& path) const
    {
        check(dsmc_out_boundary_stress_heat(h_, istep, zonemap.data(), (int32_t)zonemap.size(), path.c_str()),
              "dsmc_out_boundary_stress_heat");
        return true;
    }

    DsmcCounters counters() const
    {
        DsmcCounters c{};
        check(dsmc_get_counters(h_, &c), "dsmc_get_counters");
        return c;
    }
    void sync() const { check(dsmc_sync(h_), "dsmc_sync"); }
    DsmcHandle* handle() const { return h_; }
    int ncell() const { return ncell_; }

private:
    std::vector<double> macro(int which) const
    {
        std::vector<double> out((size_t)ncell_ * Madata);
        check(dsmc_download_macro(h_, which, out.data()), "dsmc_download_macro");
        return out;
    }
    int roleOf(int tag) const
    {
        for (int k = 0; k < params_.nzones; ++k)
            if (params_.zone_tag[k] == tag) return params_.zone_role[k];
        return DSMC_ROLE_NONE;
    }
    void check(int status, const char* what) const
    {
        if (status != DSMC_OK) throw DsmcError(std::string(what) + ": " + dsmc_last_error(h_));
    }

    DsmcHandle* h_ = nullptr;
    DsmcMeshMessage mess_{};
    DsmcCaseParams params_{};
    int ncell_ = 0, nface_ = 0;
    std::vector<DsmcEdgeRec> edges_;
};

// ProcessGSISGpu: the particle side of the reference's ProcessGSIS
// (src/ProcessGSIS.h:71-131) over a ProcessDSMCGpu: the NS solution per cell
// (nsresult, [icell][6]: density / n_ref, u, T, Tr), the DSMC->NS acceptance
// gate (dsmc2ns_macro_accepted, used when dsmc2ns_acceptance_ready) and
// molecular_velocity_change() on the device. The NS solver (MacroSolver)
// and the DSMC2NS / NS2DSMC exchanges stay with the caller, which fills
// nsresult from its NS step and reads the DSMC fields through
// ProcessDSMCGpu::local().
class ProcessGSISGpu {
public:
    explicit ProcessGSISGpu(ProcessDSMCGpu& process)
        : icell(process.ncell()), nsresult((size_t)process.ncell() * 6, 0.0),
          dsmc2ns_macro_accepted((size_t)process.ncell(), 1), process_(process)
    {
    }

    int icell;
    std::vector<double> nsresult;
    std::vector<char> dsmc2ns_macro_accepted;
    bool dsmc2ns_acceptance_ready = false;

    // molecular_velocity_change (src/ProcessGSIS.cpp:2239-2366). Where the
    // reference prints "The solution from ns solver is nan, ..." the report's
    // nan_cell is the first NaN cell (cells before it are updated, as there).
    DsmcGsisReport molecular_velocity_change()
    {
        if (nsresult.size() != (size_t)icell * 6 || dsmc2ns_macro_accepted.size() != (size_t)icell)
            throw DsmcError("molecular_velocity_change: nsresult / acceptance sizes do not match icell");
        DsmcGsisReport rep{};
        const char* gate = dsmc2ns_acceptance_ready ? dsmc2ns_macro_accepted.data() : nullptr;
        const int st = dsmc_molecular_velocity_change(process_.handle(), nsresult.data(), gate, &rep);
        if (st != DSMC_OK)
            throw DsmcError(std::string("dsmc_molecular_velocity_change: ") + dsmc_last_error(process_.handle()));
        return rep;
    }

private:
    ProcessDSMCGpu& process_;
};

}  // namespace dsmc_b200
