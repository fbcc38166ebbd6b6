"""Algorithmic DRAM bytes of the step kernel, per voxel-step.

The model counts every array the kernel must stream once per phase (s = bytes
per stored value: 4 for FP32, 8 for FP64; neighbour values are assumed to hit
in cache, as their owners stream them in the same phase):

  RHS phase  read u, h, flags, nb[6] (int32), coef[6]; write x, h', b, V0
             = 2s + 1 + 24 + 6s + 4s
  phase A_j  read V_j, nb, coef, V_0..V_{j-1}; write w           = 2s + 24 + 6s + js
  phase C_j  read w, V_0..V_j; write V_{j+1}                     = (j+3)s
  update     read x, V_0..V_{k-1}; write u (or x)                = (k+2)s
  check      read x, nb, coef, b; write V0, u (full cycles only) = 5s + 24 + 6s

A solve with k Arnoldi steps therefore costs
  B(k) = RHS + update + sum_{j<k} (A_j + C_j)
       = (13s + 25) + (k+2)s + k(11s + 24) + s k(k-1)
For FP32 this is 81 + 68 k + 4 k^2 bytes (k = 0 when the initial residual
already meets the tolerance).
"""


def bytes_rhs(s):
    return 2 * s + 1 + 24 + 6 * s + 4 * s


def bytes_iter_sum(s, k_sum, k_sq_sum):
    """sum over solves of sum_{j<k}(A_j + C_j) = sum_k [k(11s+24) + s k(k-1)]."""
    return (11 * s + 24) * k_sum + s * (k_sq_sum - k_sum)


def bytes_update(s, k_sum, solves):
    return (2 * s) * solves + s * k_sum


def bytes_check(s):
    return 5 * s + 24 + 6 * s


def algorithmic_bytes(s, voxels, steps, k_sum, k_sq_sum, checks=0):
    """Total algorithmic bytes of ``steps`` steps of an instance with ``voxels``
    voxels whose solves took ``k_sum`` Arnoldi steps in total (``k_sq_sum`` =
    sum of squares).  Steps that needed no iteration still run the RHS phase
    and the final copy (2s)."""
    per_voxel = (steps * (bytes_rhs(s) + 2 * s) + bytes_iter_sum(s, k_sum, k_sq_sum) + s * k_sum
                 + checks * bytes_check(s))
    return voxels * per_voxel


def per_voxel_step(s, k):
    return bytes_rhs(s) + 2 * s + bytes_iter_sum(s, k, k * k) + s * k
