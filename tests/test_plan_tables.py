"""Host logic without a GPU: the C++ per-direction tables (restated from
src/FFTW_plan_dim*.cpp in flups_b200/csrc/plan.cpp) equal the oracle's
(oracle/plans.py) for every BC combination and centring, and every solve of
the reference's test matrices plans its passes without error."""
import pytest

from flups_b200 import pyflups as pf
from oracle.plans import Plan, sort_plans, FORWARD, BACKWARD, CELL_CENTER, NODE_CENTER
from oracle.vtube import tube_case


def _oracle_plans(nglob, lda, bcv, h, L, center):
    out = {}
    for name, sign, green in (("fwd", FORWARD, False), ("bwd", BACKWARD, False), ("grn", FORWARD, True)):
        ps = sort_plans([Plan(1 if green else lda, d, h, L, bcv[d], sign, green, center) for d in range(3)])
        size, cplx = list(nglob), False
        for p in ps:
            if p.type == 18:
                continue
            p.init(size, cplx)
            size[p.dim] = p.n_out
            cplx = cplx or p.isr2c
        out[name] = ps
    return out


def _kind_code(k):
    if k is None:
        return 0
    fam, typ = k
    return typ if fam == "dct" else 4 + typ


def _compare(cpp, ora, lda):
    for c, o in zip(cpp, ora):
        assert c["dim"] == o.dim and c["type"] == o.type
        if o.type == 18:
            continue
        assert c["n_out"] == o.n_out and c["fieldstart"] == o.fieldstart
        assert c["isr2c"] == int(o.isr2c) and c["is_spectral"] == int(o.is_spectral)
        for key in ("koffset", "kfact", "symstart", "normfact", "volfact"):
            assert c[key] == pytest.approx(getattr(o, key), rel=1e-15, abs=0), key
        dft = o.type in (6, 8)
        for k in range(len(c["comp"])):
            cc = c["comp"][k]
            if not dft or k == 0:
                assert cc["n_in"] == o.n_in[k]
            assert (cc["fi"], cc["fo"], cc["postpro"], cc["imult"]) == (
                o.fftwstart_in[k], o.fftwstart_out[k], o.postpro[k], int(o.imult[k]))
            assert cc["kind"] == _kind_code(o.kind[k])


def _bc_matrix():
    one = [[0], [1], [4]]
    bc1 = [a + b for a in one for b in one] + [[3, 3]]
    for bx in bc1:
        for by in bc1:
            for bz in bc1 + [[9, 9]]:
                yield [bx, by, bz]


@pytest.mark.parametrize("center", [CELL_CENTER, NODE_CENTER])
def test_tables_match_oracle_over_bc_matrix(center):
    n = 0
    for bc in _bc_matrix():
        fact = 0 if center == CELL_CENTER else 1
        res = (8, 8, 1) if bc[2] == [9, 9] else (8, 8, 8)
        nglob = [res[0] + fact, res[1] + fact, 1 if res[2] == 1 else res[2] + fact]
        h = [1.0 / (nglob[0] - fact), 1.0 / (nglob[1] - fact), 1.0 if nglob[2] == 1 else 1.0 / (nglob[2] - fact)]
        bcv = [[[bc[d][0]], [bc[d][1]]] for d in range(3)]
        t = pf.Topology(0, 1, nglob)
        s = pf.Solver(t, bc, h, [1, 1, 1], center_type=[center] * 3)
        j = s.plan_json()
        o = _oracle_plans(nglob, 1, bcv, h, [1.0] * 3, center)
        for name in ("fwd", "bwd", "grn"):
            _compare(j["plans"][name], o[name], 1)
        # every pass fits the shared-memory budget of one CTA and covers its lines
        for p in j["passes"]:
            assert p["smem"] <= 227 * 1024 and p["lines_per_cta"] >= 1
        n += 1
    assert n == 1100


def test_rot_tables_per_component():
    """Per-component BCs of the vortex-tube cases (solve_vtube/src/main_vtube.cpp:140-200)."""
    for vdir in range(3):
        for sx in (0, 1, -1):
            for sy in (0, 1, -1):
                bcv, *_ = tube_case(vdir, sx, sy)
                t = pf.Topology(0, 3, [16] * 3)
                s = pf.Solver(t, [[bcv[d][0], bcv[d][1]] for d in range(3)], [1 / 16] * 3, [1, 1, 1], order_diff=1)
                j = s.plan_json(1)
                o = _oracle_plans([16] * 3, 3, bcv, [1 / 16] * 3, [1.0] * 3, CELL_CENTER)
                for name in ("fwd", "bwd"):
                    _compare(j["plans"][name], o[name], 3)
                fused = [p for p in j["passes"] if p["fused"]]
                assert len(fused) == 1 and fused[0]["comps_together"] == 1
