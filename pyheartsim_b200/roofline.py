"""Algorithmic DRAM bytes of the step kernel, per voxel-step.

Counts every array the kernel must stream once per phase; s = bytes per stored
value (4 FP32, 8 FP64), cb = coefficient bytes per row (5 for isotropic rows:
one value + a presence byte; 6 s otherwise).  Neighbour values read by the
stencil are assumed to hit in cache (their owners stream them in the same
phase).

  RHS pass 1 read u, h, flags; write h', u* (basis column 1)     = 4 s + 1
  RHS pass 2 read u*, flags, nb[6] (int32), coefficients; write x, b, V0
                                                                 = 4 s + 25 + cb
  phase A_j  read V_j, nb, coefficients, V_0..V_{j-1}; write w  = (j + 2) s + 24 + cb
  phase C_j  read w, V_0..V_j; write V_{j+1}                     = (j + 3) s
  update     read x, V_0..V_{k-1}; write u                       = (k + 2) s
  copy       (a solve that needs no iteration) read x, write u  = 2 s
  guess      (extrapolated initial guess) + s per step, + 2 s per iterated solve

A solve with k Arnoldi steps therefore costs
  B(k) = RHS + (k + 2) s + k (5 s + 24 + cb) + s k (k - 1),
e.g. 90 + 68 k + 4 k^2 bytes in FP32 with six stored coefficients, and
71 + 49 k + 4 k^2 with isotropic rows.

The plain form (GMRES(50) full cycles) also runs the true-residual test at the
end of every cycle: read x, b, nb, coefficients; write V0 and u = 4 s + 24 + cb
per cycle.

The neighbour table costs nb = 24 bytes per row as six int32 indices, or 8
with the compact table (four int16 offsets; the +-x neighbours follow from the
row order, and the per-512-voxel base offsets add 1/32 byte per row): every
"24" above becomes nb.

Anisotropic rows (edge cross terms) add the edge table, 12 int32 indices and
six coefficients = 48 + 6 s, to every operator application (the RHS stencil
and each A_j): in FP32 +72 bytes per step and +72 per Arnoldi step.
"""


def coef_bytes(s, iso):
    return (s + 1) if iso else 6 * s


COMPACT_NB = 8 + 16 / 512


def bytes_rhs(s, cb, nb=24):
    return 8 * s + 2 + nb + cb


def edge_bytes(s):
    return 48 + 6 * s


def algorithmic_bytes(s, voxels, steps, k_sum, k_sq_sum, solves=None, iso=True, guess=False, edge=False,
                      checks=0, nb=24):
    """Total algorithmic bytes of ``steps`` steps of an instance with ``voxels``
    voxels whose solves took ``k_sum`` Arnoldi steps in total (``k_sq_sum`` =
    sum of squares).  Steps that needed no iteration still run the RHS phase
    and the final copy (2 s).  ``checks``: true-residual tests at cycle ends
    (full cycles); ``nb``: neighbour-table bytes per row (24, or COMPACT_NB)."""
    cb = coef_bytes(s, iso)
    per_voxel = (steps * (bytes_rhs(s, cb, nb) + 2 * s) + (5 * s + nb + cb) * k_sum + s * (k_sq_sum - k_sum)
                 + s * k_sum + checks * (4 * s + nb + cb))
    if guess:     # read the increment in the RHS phase; read and rewrite it in the final update
        per_voxel += steps * s + 2 * s * (solves or 0)
    if edge:
        per_voxel += steps * edge_bytes(s) + edge_bytes(s) * k_sum
    return voxels * per_voxel


def per_voxel_step(s, k, iso=True, nb=24):
    return algorithmic_bytes(s, 1, 1, k, k * k, iso=iso, nb=nb)
