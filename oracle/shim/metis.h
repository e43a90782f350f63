/*
 * Stand-in for the METIS partitioner interface, used only to compile the
 * reference's own DSMC sources (oracle test infrastructure). Every cell goes
 * to part 0: the oracle runs the reference as one compute rank owning the
 * whole mesh, which is what src/meshImport.cpp:1679-1730 produces for one
 * part.
 */
#ifndef DSMC_ORACLE_METIS_STUB_H
#define DSMC_ORACLE_METIS_STUB_H

typedef int idx_t;
typedef float real_t;

#define METIS_NOPTIONS 40
#define METIS_OK 1
#define METIS_FAIL (-4)
#define METIS_OPTION_OBJTYPE 1
#define METIS_OPTION_CTYPE 2
#define METIS_OBJTYPE_CUT 0
#define METIS_CTYPE_SHEM 1

inline int METIS_SetDefaultOptions(idx_t* opts)
{
    for (int i = 0; i < METIS_NOPTIONS; ++i) opts[i] = -1;
    return METIS_OK;
}
inline int metis_stub_assign(idx_t* n, idx_t* part)
{
    for (idx_t i = 0; i < *n; ++i) part[i] = 0;
    return METIS_OK;
}
inline int METIS_PartGraphKway(idx_t* n, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*,
                               real_t*, real_t*, idx_t*, idx_t* objval, idx_t* part)
{ *objval = 0; return metis_stub_assign(n, part); }
inline int METIS_PartGraphRecursive(idx_t* n, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*, idx_t*,
                                    real_t*, real_t*, idx_t*, idx_t* objval, idx_t* part)
{ *objval = 0; return metis_stub_assign(n, part); }

#endif
