"""Class-grouped code generation of the warp-per-system layout (CPU):
the generated per-class functions, evaluated lane by lane with g++, equal
the straight-line right-hand side and Jacobian-vector product."""

import ctypes
import subprocess

import numpy as np
import pytest

from hh_models import hh_cable


def _build(nc, tmp_path):
    from cubie_b200 import create_ODE_system
    from cubie_b200.codegen import generate_system
    from cubie_b200.warpgen import generate_warp_system
    eqs, states, params, drivers = hh_cable(nc)
    sysm = create_ODE_system(eqs, states=states, parameters=params, drivers=drivers, precision=np.float64)
    w = generate_warp_system(sysm)
    g = generate_system(sysm)
    src = ("#include <cmath>\n#define __device__\n#define __forceinline__ inline\n"
           "#define CBX_NOINLINE __attribute__((noinline))\nusing std::exp; using std::pow;\n"
           + g.source + "\n" + w.source + r'''
extern "C" void eval(const double* y, const double* v, const double* p, const double* d, double t, double* f1,
                     double* f2, double* j1, double* j2, double* f3, double* j3) {
    System::dxdt<double>(y, p, d, t, f1);
    double J[System::NJ]; System::jac<double>(y, p, d, t, J); System::jmv<double>(J, v, j1);
    static double jac[WarpSystem::NNZ > 0 ? WarpSystem::NNZ : 1];
    for (int lane = 0; lane < 32; ++lane) {
        WarpSystem::dxdt_lanes<double>(y, p, d, t, f2, lane);
        WarpSystem::jmv_lanes<double>(y, v, p, d, t, j2, lane);
        WarpSystem::fj_lanes<double>(y, p, d, t, f3, jac, lane);
    }
    for (int lane = 0; lane < 32; ++lane) WarpSystem::jmv_cached<double>(v, jac, j3, lane);
}
''')
    cpp = tmp_path / "wg.cpp"
    so = tmp_path / "wg.so"
    cpp.write_text(src)
    subprocess.run(["g++", "-O1", "-shared", "-fPIC", "-o", str(so), str(cpp)], check=True, capture_output=True)
    return sysm, w, ctypes.CDLL(str(so))


@pytest.mark.parametrize("nc", [3, 40])
def test_classes_equal_straight_line_code(nc, tmp_path):
    sysm, w, L = _build(nc, tmp_path)
    assert w.n_classes_f == 6 and w.n_classes_jv <= 8      # interior, two ends, three gates
    assert "unsigned short" not in w.source                 # every index affine for this model
    N = sysm.num_states
    rng = np.random.default_rng(0)
    y = np.concatenate([rng.uniform(-80, 30, nc), rng.uniform(0, 1, 3 * nc)])
    v = rng.normal(size=N)
    p = np.array([120.0, 36.0, 0.5])
    d = np.array([3.0])
    f1, f2, j1, j2, f3, j3 = (np.zeros(N) for _ in range(6))
    ptr = lambda a: a.ctypes.data_as(ctypes.c_void_p)
    L.eval.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_double] + [ctypes.c_void_p] * 6
    L.eval(ptr(y), ptr(v), ptr(p), ptr(d), 0.0, ptr(f1), ptr(f2), ptr(j1), ptr(j2), ptr(f3), ptr(j3))
    np.testing.assert_allclose(f2, f1, rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(j2, j1, rtol=1e-12, atol=1e-10)
    # the cached Jacobian: f and J's nonzeros in one class pass, then J v
    # from the stored coefficients
    assert w.nnz == 12 * nc - 2 and w.n_classes_fj == 6
    np.testing.assert_allclose(f3, f1, rtol=1e-13, atol=1e-12)
    np.testing.assert_allclose(j3, j1, rtol=1e-12, atol=1e-10)


def test_non_affine_members_use_index_tables():
    import sympy as sp
    from cubie_b200.warpgen import group_classes
    y = sp.symbols("y0:5", real=True)
    kind = {s: ("y", i) for i, s in enumerate(y)}
    # components 0, 1 and 4 share a form; their inputs are not affine in the member index
    exprs = [y[3] ** 2, y[0] ** 2, y[1] + y[2], sp.exp(y[4]), y[2] ** 2]
    cls = group_classes(exprs, kind)
    sq = [c for c in cls if len(c.members) == 3][0]
    assert sq.members == [0, 1, 4] and [row[0] for row in sq.indices] == [3, 0, 2]
