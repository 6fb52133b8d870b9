"""ctypes wrapper of the CPU oracle (liboracle.so) -- test infrastructure only.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU baseline legs as
the checker; never by the product path.  It exposes the same entry points as
the CUDA library (prefix ``orc_`` instead of ``diva_``), so a parity test runs
one call sequence on both and compares every field.
"""
import ctypes as C
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")

LIN_DIRECT, LIN_SOR, LIN_GMRES_ILU, LIN_GMRES_WARM = 0, 1, 2, 3


def build(force=False):
    src = os.path.join(HERE, "diva_oracle.c")
    hdr = os.path.join(HERE, "..", "include", "diva.h")
    if force or not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(src), os.path.getmtime(hdr)):
        subprocess.run(["make", "-s", "-C", HERE], check=True)
    return LIB


def oracle_backend():
    import imau_ice_b200.diva as diva
    b = diva.Backend(build(), "orc_", "oracle")
    lib = b.lib
    vp = C.c_void_p
    lib.orc_set_linear_solver.argtypes = [vp, C.c_int, C.c_double, C.c_double, C.c_int, C.c_double, C.c_double]
    lib.orc_matrix.argtypes = [vp, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.POINTER(C.c_int)),
                               C.POINTER(C.POINTER(C.c_int)), C.POINTER(C.POINTER(C.c_double)),
                               C.POINTER(C.POINTER(C.c_double)), C.POINTER(C.POINTER(C.c_double))]
    for fn in ("orc_assemble_current", "orc_prepare_diva", "orc_diva_coefficients", "orc_secondary_velocities",
               "orc_3d_horizontal_velocities_diva"):
        getattr(lib, fn).argtypes = [vp]
    lib.orc_linear_iterations.argtypes = [vp]
    lib.orc_linear_iterations.restype = C.c_long
    lib.orc_calc_fraction_above_zero.argtypes = [C.c_double] * 4
    lib.orc_calc_fraction_above_zero.restype = C.c_double
    dp = C.POINTER(C.c_double)
    lib.orc_schoof2006.argtypes = [C.c_double] * 7 + [dp, dp]
    lib.orc_vertical_integrate.argtypes = [dp, C.c_int, dp]
    lib.orc_vertical_integrate.restype = C.c_double
    lib.orc_vertical_average.argtypes = [dp, C.c_int, dp]
    lib.orc_vertical_average.restype = C.c_double
    lib.orc_vertical_integration_from_bottom_to_zeta.argtypes = [dp, C.c_int, dp, dp]
    lib.orc_tridiagonal_solve.argtypes = [C.c_int, dp, dp, dp, dp]
    lib.orc_tridiagonal_solve.restype = C.c_int
    lib.orc_num_threads.restype = C.c_int
    lib.orc_set_threads.argtypes = [C.c_void_p, C.c_int32]
    lib.orc_set_threads.restype = C.c_int
    return b


def set_threads(ctx, threads):
    """OpenMP threads of the oracle's GMRES and column loops (1: the sequential algorithm
    of the parity tests; more: block-Jacobi ILU(0) over that many row blocks)."""
    ctx.backend.lib.orc_set_threads(ctx.h, int(threads))


def set_linear_solver(ctx, kind=LIN_DIRECT, rtol=1e-2, abstol=2.5, sor_nit=10000, sor_tol=2.5, sor_omega=1.3):
    """Choose the oracle's linear solver: direct (exact), SOR or GMRES(30)+ILU(0)."""
    ctx.backend.lib.orc_set_linear_solver(ctx.h, kind, rtol, abstol, sor_nit, sor_tol, sor_omega)


def matrix(ctx):
    """The CSR matrix (0-based) and vectors of the oracle's last assembly, as NumPy copies."""
    import numpy as np
    m, nnz = C.c_int(), C.c_int()
    ptr, idx = C.POINTER(C.c_int)(), C.POINTER(C.c_int)()
    val, b, x = C.POINTER(C.c_double)(), C.POINTER(C.c_double)(), C.POINTER(C.c_double)()
    ctx.backend.lib.orc_matrix(ctx.h, C.byref(m), C.byref(nnz), C.byref(ptr), C.byref(idx), C.byref(val),
                               C.byref(b), C.byref(x))
    n, z = m.value, nnz.value
    return (np.ctypeslib.as_array(ptr, (n + 1,)).copy(), np.ctypeslib.as_array(idx, (z,)).copy(),
            np.ctypeslib.as_array(val, (z,)).copy(), np.ctypeslib.as_array(b, (n,)).copy(),
            np.ctypeslib.as_array(x, (n,)).copy())
