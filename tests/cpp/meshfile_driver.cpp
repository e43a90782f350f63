// The C++ host layer's case-file reader (dsmc_b200::MeshFile in
// dig-appolo_b200/host/ProcessDSMCGpu.hpp) on the CPU: reads a Fluent case
// file, writes the DSMC arrays, the zone declarations and the mesh message
// as raw binaries, and checks that a missing file raises DsmcError.
//
//   meshfile_driver <case.cas> <outdir> <Ma> <Kn> <ppc> <L0>
#include "ProcessDSMCGpu.hpp"

#include <cstdio>
#include <iostream>
#include <string>

namespace {

bool dump(const std::string& path, const void* data, size_t bytes)
{
    FILE* f = std::fopen(path.c_str(), "wb");
    if (!f) return false;
    const bool ok = std::fwrite(data, 1, bytes, f) == bytes;
    return std::fclose(f) == 0 && ok;
}

}  // namespace

int main(int argc, char** argv)
{
    if (argc < 7) {
        std::cerr << "usage: meshfile_driver <case.cas> <outdir> <Ma> <Kn> <ppc> <L0>\n";
        return 2;
    }
    const std::string out = argv[2];
    try {
        dsmc_b200::MeshFile mesh(argv[1]);
        const DsmcMeshDesc md = mesh.desc();
        const std::vector<DsmcZone> zones = mesh.zonemap();
        const DsmcMeshMessage mm = mesh.message(std::stod(argv[3]), std::stod(argv[4]), std::stoi(argv[5]),
                                                std::stod(argv[6]));
        bool ok = dump(out + "/cells.bin", md.cells, sizeof(DsmcCellRec) * (size_t)md.ncell) &&
                  dump(out + "/edges.bin", md.edges, sizeof(DsmcEdgeRec) * (size_t)md.nface) &&
                  dump(out + "/points.bin", md.localPointXY, sizeof(double) * 3 * (size_t)md.npoint) &&
                  dump(out + "/split.bin", md.faceSplitTag, (size_t)md.nface) &&
                  dump(out + "/zones.bin", zones.data(), sizeof(DsmcZone) * zones.size()) &&
                  dump(out + "/mess.bin", &mm, sizeof mm);
        if (!ok) {
            std::cerr << "cannot write to " << out << "\n";
            return 1;
        }
    } catch (const dsmc_b200::DsmcError& e) {
        std::cerr << "unexpected DsmcError: " << e.what() << "\n";
        return 1;
    }
    try {
        dsmc_b200::MeshFile missing(out + "/no_such_case.cas");
        std::cerr << "a missing file was read\n";
        return 1;
    } catch (const dsmc_b200::DsmcError& e) {
        std::cout << "missing: " << e.what() << "\n";
    }
    std::cout << "ok\n";
    return 0;
}
