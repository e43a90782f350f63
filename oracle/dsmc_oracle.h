/*
 * dsmc_oracle.h — CPU restatement of the reference's DSMC particle step.
 *
 * ORACLE TEST INFRASTRUCTURE. Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load it, as the checker; the product never
 * calls it.
 *
 * Plain C, FP64, compiled without fused multiply-add, following
 * ProcessDSMC (src/ProcessDSMC.cpp) function by function. Random draws use
 * counter-based Philox4x32-10 streams keyed like the CUDA library's, and
 * particles are kept in the same canonical per-cell order, so an FP64 GPU
 * run can be compared with this one particle by particle; the reference's
 * own mt19937 draws are not reproducible (seeded from std::random_device at
 * src/MeshparticalInitial.h:194-198), so against the reference itself only
 * the deterministic parts (tracing, inflow counts) are compared exactly and
 * the rest statistically.
 */
#ifndef DSMC_ORACLE_H
#define DSMC_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleCase OracleCase;

/* cells/edges/mess use the byte layouts of DsmcCell / DsmcEdge / meshMessage
 * (src/meshImport.h:168-208). Roles: 0 none, 1 interface, 2 inlet,
 * 3 outlet, 4 diffuse wall, 5 specular. */
OracleCase* oracle_create(int ncell, int nface, int npoint, const void* cells, const void* edges,
                          const double* points, const unsigned char* split, const void* mess,
                          int nzones, const int* zone_tag, const int* zone_role, const int* zone_inject,
                          double dirx, double diry, int nss, int nscheme, int nevery, int nrepeat,
                          int wall_stats, uint64_t seed, int max_cross);
void oracle_destroy(OracleCase* o);

/* Philox4x32-10 of counter ctr[4] under key[2]. */
void oracle_philox(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);

/* The tracing loop of traceParticleDtleft (src/ProcessDSMC.cpp:149-221) on
 * caller-given particles; outputs as dsmc_trace(). */
void oracle_trace(OracleCase* o, int64_t n, const double* px, const double* py, const double* pz,
                  const double* vx, const double* vy, const double* vz, const double* dt, const int* cell,
                  int stop_at_wall, int* out_cell, int* out_ifout, int* out_face, int* out_tri, int* out_ncross,
                  double* out_px, double* out_py, double* out_pz, double* out_vx, double* out_vy,
                  double* out_vz, double* out_dt);

/* Particle store (cell-major, input order within a cell). */
int oracle_set_particles(OracleCase* o, int64_t n, const double* px, const double* py, const double* pz,
                         const double* vx, const double* vy, const double* vz, const double* ir, const int* cell);
int64_t oracle_count(const OracleCase* o);
void oracle_get_particles(const OracleCase* o, double* px, double* py, double* pz, double* vx, double* vy,
                          double* vz, double* ir, int* cell);

/* One step, stage flags as DSMC_STAGE_* of include/dsmc_gpu.h. */
int oracle_step(OracleCase* o, int istep, unsigned stages);
void oracle_macro_pre(OracleCase* o);

void oracle_get_macro(OracleCase* o, int which, double* out);   /* 0 local, 1 record, 2 final_record */
void oracle_get_step_moments(const OracleCase* o, double* out); /* [ncell][18] */
void oracle_get_acc(const OracleCase* o, double* out);          /* [ncell][54] */
void oracle_get_cell_state(const OracleCase* o, double* crmax, double* rem_coll, double* rem_inj);
void oracle_set_cell_state(OracleCase* o, const double* crmax, const double* rem_coll, const double* rem_inj);
/* dsmc2ns_sparse_state as the host's GSIS exchange writes it back
 * (src/ProcessGSIS.cpp:1660-1674); values outside 0..2 return -1. */
int oracle_set_sparse_state(OracleCase* o, const unsigned char* sparse_state);
void oracle_get_counts(const OracleCase* o, int* ppc, double* window_samples, char* window_valid,
                       unsigned char* sparse_state);
void oracle_get_wall(const OracleCase* o, double* tally);        /* [nface][6] */
/* injected, removed, dropped, lost, wall_hits, crossings, pairs, collisions */
void oracle_counters(const OracleCase* o, uint64_t out[8]);
/* Placement tetrahedra (buildCellInitTets): off[ncell+1], V[nplace*12],
 * vol[nplace] (any may be NULL); returns nplace. */
int oracle_placement(const OracleCase* o, int* off, double* V, double* vol);
/* Initial fill as dsmc_fill_initial (at_rest = 1) / dsmc_fill_freestream. */
int oracle_fill(OracleCase* o, double ppc_mean, uint64_t seed, int at_rest);
/* GSIS particle update as dsmc_molecular_velocity_change; report: nan cell,
 * cells updated, cells skipped, added, removed, particles. */
int oracle_molecular_velocity_change(OracleCase* o, const double* ns, const char* accepted, int64_t report[6]);

#ifdef __cplusplus
}
#endif
#endif
