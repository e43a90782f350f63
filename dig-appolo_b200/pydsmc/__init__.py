"""Host-side helpers of the B200 DSMC step: synthetic meshes in the
reference's format (mesh), case constants (case), seeded inputs (workload)
and the ctypes binding of the C ABI (gpu)."""
