/*
 * dsmc_meshio.h — native mesh input and field output of the B200 DSMC
 * library (libdsmcgpu.so): the Fluent ASCII case reader and the DSMC
 * topology builder that turn a CAS file into the arrays dsmc_create takes,
 * the case constants (meshMessage), and the Fluent data writers of the
 * sampled cell fields and the wall fields.
 *
 * Conventions as dsmc_gpu.h: extern "C", plain pointers and sizes, 0 or a
 * negative DSMC_E_* status. Functions without a handle leave their message
 * in dsmc_meshio_last_error() (per host thread). Host code only: nothing
 * here needs a GPU.
 */
#ifndef DSMC_MESHIO_H
#define DSMC_MESHIO_H

#include "dsmc_gpu.h"

#ifdef __cplusplus
extern "C" {
#endif

/* faceSplitTag values (meshImport::FACE_SPLIT_*, src/meshImport.h:309-327):
 * the quad's triangles are (0,1,2)+(0,2,3), (0,1,3)+(1,2,3), or none. */
#define DSMC_FACE_SPLIT_02 0
#define DSMC_FACE_SPLIT_13 1
#define DSMC_FACE_SPLIT_INVALID 255

/* A mesh read from a Fluent ASCII case file, owned by the library. */
typedef struct DsmcMeshFile DsmcMeshFile;

/* One zone declaration of the case file, in file order (ZONE,
 * src/meshImport.h:120-129, filled by meshImport::getZoneid,
 * src/meshImport.cpp:524-551). section 12: a cell zone, 13: a face zone;
 * first / last are 1-based indices. */
typedef struct DsmcZone {
    int32_t section;
    int32_t id;
    int32_t first;
    int32_t last;
} DsmcZone;

/* Read a Fluent ASCII case and build the DSMC arrays for one partition
 * (replaces meshImport::meshImport(path, nParts, 1) + readCAS + setFaceCellNew
 * + preprocess, src/meshImport.cpp:35-41, 177-849, and the DSMC topology of
 * rootCaptureGlobalDsmcAndReleaseMesh with choose_face_level_quad_split_tag,
 * src/meshImportDsmcTopology.cpp:85-228):
 *   - sections (2 dim), (10 nodes), (12 cells), (13 faces) as readCAS
 *     classifies them (hexadecimal indices, 1-based; a face's second cell 0
 *     marks a boundary face, which gets a ghost id Ncell, Ncell+1, ... in
 *     file order; zone headers recorded as DsmcZone); other sections are
 *     skipped; hexadecimal digits may be upper or lower case;
 *   - face centroid, area and unit normal from the fan of triangles about
 *     the node average; cell2face / cell2cell / cell2face_sgn in face
 *     order; cell volume and centroid from the face pyramids; normals
 *     oriented from c0 to c1 (ghost centroids mirrored through the face);
 *   - quad faces split along the diagonal whose two triangles are flatter
 *     and closer in area (ties to 0-2).
 * All floating-point operations in the reference's order, without fused
 * multiply-add: the arrays equal the reference's bit for bit. *out is NULL
 * on failure (unreadable file, a cell with more than 6 faces, indices out
 * of range). */
int dsmc_mesh_read_cas(const char* path, DsmcMeshFile** out);
void dsmc_mesh_free(DsmcMeshFile* m);
const char* dsmc_meshio_last_error(void);

/* The arrays dsmc_create takes; the pointers stay valid until
 * dsmc_mesh_free. */
int dsmc_mesh_get_desc(const DsmcMeshFile* m, DsmcMeshDesc* md);

/* Zone declarations in file order: *count is set to the number of zones;
 * at most capacity are copied into zones (which may be NULL). */
int dsmc_mesh_get_zones(const DsmcMeshFile* m, DsmcZone* zones, int32_t capacity, int32_t* count);

/* Summed cell volumes (meshImport::Area), the shortest face edge
 * (meshImport::miniLength, from setParticleMessage) and the number of
 * boundary faces (bcnumber). Any pointer may be NULL. */
int dsmc_mesh_get_stats(const DsmcMeshFile* m, double* area_sum, double* min_edge, int32_t* bcnumber);

/* meshMessage of the mesh (setMa_Kn_CFL, setMeshMessage and
 * setParticleMessage, src/meshImport.cpp:1252-1405): the constants the
 * reference hard-codes are arguments (its values: L0 = 3.912 m, T_in =
 * 142.2 K, T_wall = 300 K at src/meshImport.cpp:1316-1318, ppc = 100 at
 * src/meshImport.h:47; cfl = 1e2 and cfl_ns = 5 from main's setMa_Kn_CFL
 * call). Neff = Area n_ref / (ppc Ncell), dtime = 0.2 miniLength. */
int dsmc_mesh_message(const DsmcMeshFile* m, double Ma, double Kn, int32_t ppc, double L0, double T_in,
                      double T_wall, double cfl, double cfl_ns, DsmcMeshMessage* out);

/* meshImport::out2Fluent_dsmc (src/meshImport.cpp:1107-1182): the Fluent
 * data sections 700 (density), 701 (velocity / (sqrt(gamma/2) v_in/v_rms)),
 * 702 (T, Tr / (T_in/T_ref)), 710 (stress / (T_in/T_ref)), 711 and 712
 * (heat fluxes / both scales) of the cell zone with id 2, one line per cell
 * in the reference's text format (six significant digits). w is
 * [ncell][18] in MacroIndex order (out2dat's selection of record or
 * final_record: dsmc_out2dat does it). Fails when no cell zone has id 2 or
 * its range exceeds ncell. */
int dsmc_write_fluent_cells(const char* path, const DsmcMeshMessage* mess, const DsmcZone* zones, int32_t nzones,
                            const double* w, int32_t ncell);

/* The wall-field file of ProcessDSMC::outBoundaryStressHeat
 * (src/ProcessDSMC.cpp:3451-3652): per face of the diffuse-wall zones (zone
 * roles from params), pressure, shear, stress vector, normal and
 * translational / rotational / total heat flux from the steady tallies
 * tally [nface][6] (hits, momentum change (3), translational and rotational
 * energy change; dsmc_download_wall) scaled by 2 Neff / (dt (istep - nss))
 * / area / n_ref (one step's worth until istep passes nss); written as
 * sections 700-706 for every zone declaration whose face range holds only
 * wall faces, 16 significant digits. Writes nothing and returns 0 when no
 * zone qualifies. The reference's build turns this output off
 * (EnableBoundaryStressHeatStatistic, src/meshImport.h:51); here it is
 * written whenever called. */
int dsmc_write_fluent_wall(const char* path, const DsmcMeshMessage* mess, const DsmcCaseParams* params,
                           const DsmcZone* zones, int32_t nzones, const DsmcEdgeRec* edges, int32_t nface,
                           const double* tally, int32_t istep);

/* ProcessDSMC::out2dat(istep) (src/ProcessDSMC.cpp:3338-3438) for a case on
 * the device: record up to NSS and for sparse cells (states 1, 2),
 * final_record after, written with dsmc_write_fluent_cells. The reference
 * names the file ./statisticResults/DSMCKn%.1f_iter%d_CELL%d.dat (Kn,
 * istep, Ncell); here the caller gives the path. */
int dsmc_out2dat(DsmcHandle* h, int32_t istep, const DsmcZone* zones, int32_t nzones, const char* path);

/* ProcessDSMC::outBoundaryStressHeat(istep) for a case on the device: the
 * wall tallies (wall_stats on) written with dsmc_write_fluent_wall. The
 * reference names the file
 * ./statisticResults/BoundaryStressHeatFluentKn%.1f_iter%d.dat. */
int dsmc_out_boundary_stress_heat(DsmcHandle* h, int32_t istep, const DsmcZone* zones, int32_t nzones,
                                  const char* path);

#ifdef __cplusplus
}
#endif

#endif
