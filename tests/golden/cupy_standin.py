"""NumPy/SciPy stand-in for the parts of CuPy the reference calls.

Test infrastructure only: ``make_golden.py`` installs this module as
``cupy``/``cupyx.scipy.sparse``/``cupyx.scipy.sparse.linalg`` so that the
reference's own ``simulation/simulation_gpu.py`` runs unmodified under
``NUMBA_ENABLE_CUDASIM=1`` in a container without CuPy or a GPU.

The GMRES below restates the documented behaviour of
``cupyx.scipy.sparse.linalg.gmres`` (CuPy 12-13, ``_iterative.py``), the solver
the reference calls at simulation/simulation_gpu.py:253:

* ``atol_eff = max(atol, tol * ||b||)``; ``||b|| == 0`` returns ``b``;
* each cycle starts with the true residual ``r = b - A x``; the solve stops when
  ``||r|| <= atol_eff`` or ``iters >= maxiter``;
* otherwise one FULL Arnoldi cycle of ``restart`` steps with classical
  Gram-Schmidt (``h = V^T u``, ``u -= V h``, one pass, no re-orthogonalisation,
  no breakdown test), the ``(restart+1) x restart`` Hessenberg least-squares
  solved on the host with ``numpy.linalg.lstsq`` and ``x += V y``;
* the iterate returned is the one whose residual passed the test.

``FLOAT`` selects the storage dtype (float32 as shipped, float64 for the FP64
golden runs) in the same way CuPy follows the matrix dtype.
"""
import numpy as _np
import scipy.sparse as _sp

float32 = _np.float32
float64 = _np.float64
int32 = _np.int32


def zeros(shape, dtype=float):
    return _np.zeros(shape, dtype=dtype)


def asarray(a, dtype=None):
    return _np.array(a, dtype=dtype, copy=True)


def array(a, dtype=None):
    return _np.array(a, dtype=dtype, copy=True)


def asnumpy(a):
    return _np.array(a, copy=True)


class _Sparse:
    @staticmethod
    def coo_matrix(arg, shape=None):
        return _sp.coo_matrix(arg, shape=shape)

    @staticmethod
    def identity(n, format='csr', dtype=float):
        return _sp.identity(n, format=format, dtype=dtype)


sparse = _Sparse()


def gmres(A, b, x0=None, tol=1e-5, restart=None, maxiter=None, M=None,
          callback=None, atol=None, callback_type=None, rtol=None):
    if rtol is not None:
        tol = rtol
    dtype = A.dtype
    n = A.shape[0]
    b = _np.asarray(b).astype(dtype).ravel()
    x = (_np.zeros(n, dtype) if x0 is None else _np.asarray(x0).astype(dtype).ravel())
    if n == 0:
        return _np.empty_like(b), 0
    b_norm = _np.linalg.norm(b)
    if b_norm == 0:
        return b, 0
    atol = tol * float(b_norm) if atol is None else max(float(atol), tol * float(b_norm))
    maxiter = n * 10 if maxiter is None else maxiter
    restart = 20 if restart is None else restart
    restart = min(restart, n)
    V = _np.empty((n, restart), dtype=dtype, order='F')
    H = _np.zeros((restart + 1, restart), dtype=dtype, order='F')
    e = _np.zeros((restart + 1,), dtype=_np.float64)
    iters = 0
    while True:
        mx = x
        r = b - A @ mx
        r_norm = _np.linalg.norm(r)
        if r_norm <= atol or iters >= maxiter:
            break
        v = r / r_norm
        V[:, 0] = v
        e[0] = r_norm
        for j in range(restart):
            u = A @ v
            h = V[:, :j + 1].T @ u
            u = u - V[:, :j + 1] @ h
            H[:j + 1, j] = h
            H[j + 1, j] = _np.linalg.norm(u)
            if j + 1 < restart:
                v = u / H[j + 1, j]
                V[:, j + 1] = v
        y = _np.linalg.lstsq(H, e, rcond=None)[0]
        x += (V @ y).astype(dtype)
        iters += restart
    info = 0
    if iters == maxiter and not (r_norm <= atol):
        info = iters
    return mx, info


def cg(A, b, x0=None, tol=1e-5, maxiter=None, M=None, callback=None, atol=None):
    raise NotImplementedError("the reference never calls cg (method='gmres' is hard-coded)")
