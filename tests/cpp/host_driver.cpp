// Test driver for the C++ host layer (dig-appolo_b200/host/ProcessDSMCGpu.hpp).
//
// Reads a case written by tests/test_gpu_host_cpp.py (raw arrays in the C-ABI
// layouts), runs it through ProcessDSMCGpu the way the reference's main loop
// drives ProcessDSMC (src/meshImportTest.cpp:207-234) and writes the
// particles, the macro fields and the wall fields back for comparison.
//
//   host_driver <dir> <nsteps> <mode: 0 stage calls, 1 fused step,
//                                    2 fused steps, then a GSIS particle
//                                    update from <dir>/ns.bin and <dir>/acc.bin
//                                    and one more step>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "ProcessDSMCGpu.hpp"

template <typename T>
static std::vector<T> load(const std::string& path, size_t n)
{
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    if (!f.read(reinterpret_cast<char*>(v.data()), (std::streamsize)(n * sizeof(T))))
        throw std::runtime_error("cannot read " + path);
    return v;
}

template <typename T>
static void save(const std::string& path, const std::vector<T>& v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), (std::streamsize)(v.size() * sizeof(T)));
}

int main(int argc, char** argv)
{
    if (argc < 4) {
        std::cerr << "usage: host_driver <dir> <nsteps> <mode>\n";
        return 2;
    }
    const std::string d = argv[1];
    const int nsteps = std::stoi(argv[2]);
    const int mode = std::stoi(argv[3]);
    const int fused = mode != 0;
    try {
        std::ifstream meta(d + "/case.txt");
        long ncell, nface, npoint, n;
        meta >> ncell >> nface >> npoint >> n;
        const auto cells = load<DsmcCellRec>(d + "/cells.bin", (size_t)ncell);
        const auto edges = load<DsmcEdgeRec>(d + "/edges.bin", (size_t)nface);
        const auto pts = load<double>(d + "/points.bin", (size_t)npoint * 3);
        const auto split = load<unsigned char>(d + "/split.bin", (size_t)nface);
        const auto mess = load<DsmcMeshMessage>(d + "/mess.bin", 1);
        const auto params = load<DsmcCaseParams>(d + "/params.bin", 1);
        DsmcMeshDesc md{};
        md.ncell = (int32_t)ncell; md.nface = (int32_t)nface; md.npoint = (int32_t)npoint;
        md.cells = cells.data(); md.edges = edges.data(); md.localPointXY = pts.data(); md.faceSplitTag = split.data();

        dsmc_b200::ProcessDSMCGpu process(md, mess[0], params[0], 0);
        dsmc_b200::Particles p;
        p.x = load<double>(d + "/x.bin", (size_t)n); p.y = load<double>(d + "/y.bin", (size_t)n);
        p.z = load<double>(d + "/z.bin", (size_t)n); p.vx = load<double>(d + "/vx.bin", (size_t)n);
        p.vy = load<double>(d + "/vy.bin", (size_t)n); p.vz = load<double>(d + "/vz.bin", (size_t)n);
        p.ir = load<double>(d + "/ir.bin", (size_t)n); p.cell = load<int32_t>(d + "/cell.bin", (size_t)n);
        process.uploadParticles(p);
        process.statistic_macroPre();
        for (int istep = 1; istep <= nsteps; ++istep) {
            if (fused) {
                process.step(istep);
            } else {
                process.preprocesseffquad(istep);
                process.advection(istep);
                process.cache2chain();
                process.collisionDSMC();
                process.statistic_macro(istep);
            }
        }
        if (mode == 2) {
            dsmc_b200::ProcessGSISGpu gsis(process);
            gsis.nsresult = load<double>(d + "/ns.bin", (size_t)ncell * 6);
            gsis.dsmc2ns_macro_accepted = load<char>(d + "/acc.bin", (size_t)ncell);
            gsis.dsmc2ns_acceptance_ready = true;
            const DsmcGsisReport rep = gsis.molecular_velocity_change();
            std::ofstream(d + "/out_gsis.txt") << rep.nan_cell << ' ' << rep.cells_updated << ' ' << rep.cells_skipped
                                               << ' ' << rep.added << ' ' << rep.removed << ' ' << rep.particles << '\n';
            process.step(nsteps + 1);
        }
        const dsmc_b200::Particles q = process.downloadParticles();
        for (const char* k : {"x", "y", "z", "vx", "vy", "vz", "ir"}) {
            const std::string s(k);
            const std::vector<double>& v = s == "x" ? q.x : s == "y" ? q.y : s == "z" ? q.z : s == "vx" ? q.vx
                                         : s == "vy" ? q.vy : s == "vz" ? q.vz : q.ir;
            save(d + "/out_" + s + ".bin", v);
        }
        save(d + "/out_cell.bin", q.cell);
        save(d + "/out_local.bin", process.local());
        save(d + "/out_record.bin", process.record());
        save(d + "/out_final.bin", process.final_record());
        save(d + "/out_out2dat.bin", process.out2datFields(nsteps));
        if (!process.outBoundaryStressHeat(nsteps, d + "/out_wall.dat")) throw std::runtime_error("wall output");
        if (!process.out2dat(nsteps, d + "/out_fluent.dat")) throw std::runtime_error("field output");
        // an invalid call reports through the exception, like a failed
        // reference call reports through its abort message
        bool threw = false;
        try {
            std::vector<DsmcCaseParams> bad = params;
            bad[0].nzones = -1;
            dsmc_b200::ProcessDSMCGpu broken(md, mess[0], bad[0], 0);
        } catch (const dsmc_b200::DsmcError& e) {
            threw = true;
            std::ofstream(d + "/out_error.txt") << e.what() << "\n";
        }
        if (!threw) throw std::runtime_error("invalid parameters were accepted");
        const DsmcCounters c = process.counters();
        std::ofstream(d + "/out_counters.txt") << c.steps << ' ' << c.injected << ' ' << c.collisions << '\n';
    } catch (const std::exception& e) {
        std::cerr << "host_driver: " << e.what() << "\n";
        return 1;
    }
    return 0;
}
