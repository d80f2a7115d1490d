"""The advanced spectral API (flups_get_innerBuffer, flups_get_innerTopo_*,
flups_do_copy / do_FFT / do_mult, src/flups.h:473-578) through the C ABI:
copy, forward transforms, Green's multiply and backward transforms must
reproduce flups_solve (STD and ROT), forward then backward must return the
input divided by the solver's normalisation, and a user-side spectral filter
written like the reference's solve_advanced sample (host loops over the inner
buffer with flups_get_spectralInfo and the symmetric index) must give the
analytic result on a periodic sine mode."""
import numpy as np
import pytest

from gpu_helpers import make_solver, to_user
from oracle.plans import CELL_CENTER, NODE_CENTER, CHAT_2, HEJ_2

pytestmark = pytest.mark.gpu

FWD, BWD, BWD_DIFF = -1, 1, 2


def _adv_solve(s, t, u, typ=0):
    inner = s.get_inner_buffer()
    s.do_copy(t, u, FWD)
    s.do_fft(inner, FWD)
    s.do_mult(inner, typ)
    s.do_fft(inner, BWD_DIFF if typ == 1 else BWD)
    out = np.zeros_like(u)
    s.do_copy(t, out, BWD)
    return out


@pytest.mark.parametrize("nglob,bcv,center,kernel", [
    ([48] * 3, [[[4], [4]]] * 3, CELL_CENTER, HEJ_2),
    ([17, 9, 9], [[[0], [1]], [[3], [3]], [[4], [4]]], NODE_CENTER, CHAT_2),
])
def test_advanced_equals_solve(nglob, bcv, center, kernel):
    fact = 0 if center == CELL_CENTER else 1
    h = [1.0 / (nglob[0] - fact)] * 3
    L = [h[d] * (nglob[d] - fact) for d in range(3)]
    t, s = make_solver(nglob, 1, bcv, h, L, center, kernel)
    u = to_user(np.random.default_rng(1).standard_normal((1,) + tuple(nglob)))
    ref = np.zeros_like(u)
    s.solve(ref, u)
    got = _adv_solve(s, t, u)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12
    if center != CELL_CENTER:
        return  # node-centred ODD / PER boundary nodes are imposed, not transformed back
    # forward then backward: the input over the normalisation
    inner = s.get_inner_buffer()
    s.do_copy(t, u, FWD)
    s.do_fft(inner, FWD)
    s.do_fft(inner, BWD)
    back = np.zeros_like(u)
    s.do_copy(t, back, BWD)
    nf = s.plan_json()["normfact"]
    assert np.linalg.norm(back * nf - u) / np.linalg.norm(u) <= 1e-12
    assert s.last_error() == 0


def test_advanced_rot_equals_solve():
    n = 32
    t, s = make_solver([n] * 3, 3, [[[4] * 3, [4] * 3]] * 3, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, HEJ_2, odiff=1)
    u = to_user(np.random.default_rng(2).standard_normal((3, n, n, n)))
    ref = np.zeros_like(u)
    s.solve(ref, u, 1)
    got = _adv_solve(s, t, u, typ=1)
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= 1e-12


def test_spectral_filter_like_the_sample():
    n = 32
    t, s = make_solver([n] * 3, 1, [[[3], [3]]] * 3, [1.0 / n] * 3, [1.0] * 3, CELL_CENTER, CHAT_2)
    x = (np.arange(n) + 0.5) / n
    X, Y, Z = np.meshgrid(x, x, x, indexing="ij")
    f = np.sin(2 * np.pi * X) * np.sin(2 * np.pi * Y) * np.sin(2 * np.pi * Z)
    u = to_user(f[None])
    inner = s.get_inner_buffer()
    s.do_copy(t, u, FWD)
    s.do_fft(inner, FWD)
    s.do_mult(inner, 0)
    # host loops over the spectral topology, as main_solve_advanced.c does
    ts = s.get_inner_topo_spectral()
    kf, ko, ss = s.get_spectral_info()
    ax0 = ts.axis
    nmem = [ts.get_nmem(d) for d in range(3)]
    nloc = [ts.get_nloc(d) for d in range(3)]
    assert ts.is_complex

    def sym(i, d):
        if ss[d] == 0.0 or i <= ss[d]:
            return i
        return -max(int(abs(2.0 * ss[d] - i)), 1)

    sig = 1e-3
    k = [np.array([(sym(i, d) + ko[d]) * kf[d] for i in range(nloc[d])]) for d in range(3)]
    ksq = k[0][:, None, None] ** 2 + k[1][None, :, None] ** 2 + k[2][None, None, :] ** 2   # [i0][i1][i2]
    view = inner[: 2 * nmem[0] * nmem[1] * nmem[2]].reshape(nmem[2], nmem[1], nmem[0], 2)
    filt = np.exp(-sig * ksq).transpose(2, 1, 0)[:, :, :, None]
    assert ax0 == 0
    view[: nloc[2], : nloc[1], : nloc[0]] *= filt
    s.do_fft(inner, BWD)
    out = np.zeros_like(u)
    s.do_copy(t, out, BWD)
    k2 = 3 * (2 * np.pi) ** 2
    exact = -np.exp(-sig * k2) / k2 * u
    assert np.linalg.norm(out - exact) / np.linalg.norm(exact) <= 1e-12


@pytest.mark.parametrize("nglob,precision", [([32, 384, 32], 32), ([384, 32, 32], 32), ([32, 384, 32], 64),
                                             ([48, 40, 36], 32), ([64] * 3, 64)])
def test_forward_spectrum_matches_numpy(nglob, precision):
    """The forward transforms alone (flups_do_FFT) against numpy: an all-unbounded
    cell-centred field is zero-padded to twice its size and transformed (r2c in
    x, c2c in y and z).  Unlike a solve, this checks each transform on its own,
    so an error that a forward / inverse pair would undo cannot hide (768-point
    lines: first radix 48 in FP32 rows and columns)."""
    nx, ny, nz = nglob
    h = [1.0 / nx] * 3
    t, s = make_solver(nglob, 1, [[[4], [4]]] * 3, h, [h[d] * nglob[d] for d in range(3)], CELL_CENTER, HEJ_2,
                       precision=precision)
    f = np.random.default_rng(7).standard_normal((nx, ny, nz))
    u = to_user(f[None])
    inner = s.get_inner_buffer()
    s.do_copy(t, u, FWD)
    s.do_fft(inner, FWD)
    ts = s.get_inner_topo_spectral()
    nmem = [ts.get_nmem(d) for d in range(3)]
    nloc = [ts.get_nloc(d) for d in range(3)]
    assert nloc == [nx + 1, 2 * ny, 2 * nz]
    view = inner[: 2 * nmem[0] * nmem[1] * nmem[2]].reshape(nmem[2], nmem[1], nmem[0], 2)
    got = view[: nloc[2], : nloc[1], : nloc[0], 0] + 1j * view[: nloc[2], : nloc[1], : nloc[0], 1]
    a = np.zeros((2 * nz, 2 * ny, 2 * nx))
    a[:nz, :ny, :nx] = f.transpose(2, 1, 0)
    ref = np.fft.fft(np.fft.fft(np.fft.rfft(a, axis=2), axis=1), axis=0)
    tol = 2e-6 if precision == 32 else 1e-12
    assert np.linalg.norm(got - ref) / np.linalg.norm(ref) <= tol
    assert s.last_error() == 0
