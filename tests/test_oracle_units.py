"""Oracle unit checks pinned to the reference's own unit-test values."""
import numpy as np
import pytest

from oracle import elem, inp


def test_lut_interpolation():
    # src/solver/material.rs:285-295
    lut = inp.LUT()
    for t, v in [(0.0, 100.0), (100.0, 200.0), (200.0, 400.0)]:
        lut.push(t, v)
    t = np.array([d[0] for d in lut.data]); v = np.array([d[1] for d in lut.data])
    for temp, want in [(-10, 100), (0, 100), (50, 150), (100, 200), (150, 300), (200, 400), (250, 400)]:
        assert lut.interpolate(temp) == want
        assert elem.lut_interp(t, v, temp) == want


def test_base_material_elastic():
    # src/solver/material.rs:299-319
    e = inp.LUT(); nu = inp.LUT()
    e.push(0.0, 210000.0); e.push(500.0, 150000.0)
    nu.push(0.0, 0.3); nu.push(500.0, 0.35)
    assert e.interpolate(0.0) == 210000.0 and nu.interpolate(0.0) == 0.3
    assert e.interpolate(250.0) == 180000.0
    assert abs(nu.interpolate(250.0) - 0.325) < 1e-12


def test_amplitude_interpolate():
    # src/solver/amplitude.rs:108-141
    ts, vs = [0.0, 10.0, 20.0], [0.0, 100.0, 200.0]
    f = inp.amplitude_interpolate
    assert abs(f(10.0, ts, vs, 0.0, 0.0) - 100.0) < 1e-15
    assert abs(f(5.0, ts, vs, 0.0, 0.0) - 50.0) < 1e-15
    assert abs(f(15.0, ts, vs, 5.0, 20.0) - 120.0) < 1e-15
    assert f(-10.0, ts, vs, 0.0, 0.0) == 0.0 and f(30.0, ts, vs, 0.0, 0.0) == 200.0


def test_preprocess_and_arguments():
    # src/solver/parser.rs:951-971
    raw = "**comment\n word  \n \t*keyword\n123.4\n4, 5, 6,\n7, 8, 9"
    assert inp.preprocess_inp(raw) == "WORD\n*KEYWORD\n123.4\n4, 5, 6, 7, 8, 9\n"
    assert inp.keyword_arguments("*STEP , INC =  100")["INC"] == "100"
    assert inp.positional_arguments("0.1, 1, 1E-05, 0.2") == ["0.1", "1", "1E-05", "0.2"]
    assert "DIRECT" in inp.preprocess_inp("*Static, Solver=Spooles") and \
        "ITERATIVE" in inp.preprocess_inp("*static, solver=iterative scaling")
    # substitute_ccx_solvers (parser.rs:930-942) is one aho-corasick replace_all pass:
    # a replacement never forms a new match
    assert inp.substitute_ccx_solvers("ITERATIVE CHOLESKY SCALING") == "ITERATIVE SCALING"
    assert inp.substitute_ccx_solvers("SPOOLESPOOLES PASTIX PARDISO") == "DIRECTPOOLES DIRECT DIRECT"


def test_c3d20_shape_functions():
    # src/solver/mesh_lib/elements/c3d20.rs:243-266, plus derivative consistency
    for p in [(0.0, 0.0, 0.0), (0.5, -0.3, 0.8)]:
        n, _ = elem.shape_c3d20(*p)
        assert abs(n.sum() - 1.0) < 1e-12
    n, _ = elem.shape_c3d20(-1.0, -1.0, -1.0)
    assert abs(n[0] - 1.0) < 1e-12 and np.all(np.abs(n[1:]) < 1e-12)
    n, _ = elem.shape_c3d20(0.0, -1.0, -1.0)
    assert abs(n[8] - 1.0) < 1e-12
    rng = np.random.default_rng(0)
    for _ in range(5):
        p = rng.uniform(-1, 1, 3)
        _, dn = elem.shape_c3d20(*p)
        assert abs(dn.sum(axis=1)).max() < 1e-12
        h = 1e-6
        for d in range(3):
            q1, q2 = p.copy(), p.copy(); q1[d] += h; q2[d] -= h
            fd = (elem.shape_c3d20(*q1)[0] - elem.shape_c3d20(*q2)[0]) / (2 * h)
            assert np.abs(fd - dn[d]).max() < 1e-8


def test_gauss_rules():
    pts, w = elem.gauss_points(20)
    assert pts.shape == (27, 3) and abs(w.sum() - 8.0) < 1e-12
    assert tuple(pts[1]) == (-0.774596669241483, -0.774596669241483, 0.0)  # zeta innermost
    pts, w = elem.gauss_points(4)
    assert pts.shape == (1, 3) and abs(w[0] - 1 / 6) < 1e-15


MAT_DECK = """
*MATERIAL, NAME=TestMat
*DENSITY
1000.0, 0.0
900.0, 500.0
*ELASTIC
210000.0, 0.3, 0.0
150000.0, 0.35, 500.0
"""

THERM_DECK = """
*MATERIAL, NAME=ThermalMat
*EXPANSION, ZERO=20.0
1.2E-5, 0.0
1.5E-5, 500.0
*INITIAL CONDITIONS, TYPE=TEMPERATURE
1, 100.0
"""


def test_material_parsing():
    # tests/material_parsing.rs:5-36
    p = inp.parse_inp_text(MAT_DECK)
    assert len(p.materials) == 1 and p.materials[0].name == "TESTMAT"
    m = p.materials[0]
    assert [m.density.interpolate(t) for t in (0, 250, 500, 600)] == [1000.0, 950.0, 900.0, 900.0]
    assert m.youngs_modulus.interpolate(250.0) == 180000.0
    assert abs(m.poisson_ratio.interpolate(250.0) - 0.325) < 1e-12


def test_thermal_parsing():
    # tests/material_parsing.rs:38-60
    p = inp.parse_inp_text(THERM_DECK)
    m = p.materials[0]
    assert m.reference_temperature == 20.0
    assert m.thermal_expansion.interpolate(0.0) == 1.2e-5
    assert m.thermal_expansion.interpolate(250.0) == 1.35e-5
    assert m.thermal_expansion.interpolate(500.0) == 1.5e-5
    assert p.initial_temperatures[1] == 100.0


def test_parser_errors_and_quirks():
    with pytest.raises(inp.FerrixError) as ei:
        inp.parse_inp_text("*ORIENTATION, NAME=X\n")
    assert ei.value.kind == "UnsupportedKeyword"
    with pytest.raises(inp.FerrixError) as ei:
        inp.parse_inp_text("*STEP\n*STATIC, SOLVER=MAGIC\n")
    assert ei.value.kind == "UnknownSolver"
    deck = ("*NODE\n1,0,0,0\n2,1,0,0\n*NSET, NSET=A\n1, 2\n*STEP\n*STATIC\n"
            "*BOUNDARY\nA, 1, 6, 0\n2, 2, 2, 0\n*CLOAD\nA, 3, 5.0\n*NODE PRINT\nU\n*CLOAD\n2, 1, 1.0\n*END STEP\n")
    p = inp.parse_inp_text(deck)
    s = p.steps[0]
    # only the first *BOUNDARY data line is read; DOFs 4-6 dropped
    assert [(b.node_id, b.dof) for b in s.bcs] == [(1, 0), (1, 1), (1, 2), (2, 0), (2, 1), (2, 2)]
    # nset CLOAD gives the full value to every node; second *CLOAD continues after *NODE PRINT
    assert [(l.node_id, l.dof, l.value) for l in s.loads] == [(1, 2, 5.0), (2, 2, 5.0), (2, 0, 1.0)]


# ---- result fields (oracle/stress.py) ------------------------------------------------------------

def test_stress_oracle_c3d20_derivatives_match_the_c_restatement():
    from oracle import elem, stress
    rng = np.random.default_rng(3)
    pts = list(stress.C3D20_NODES) + list(rng.uniform(-1, 1, size=(5, 3)))
    for q in pts:
        g = stress.c3d20_local_derivatives(np.asarray(q, dtype=np.float64))
        _, dn = elem.shape_c3d20(*q)
        assert np.abs(g - dn).max() < 1e-14
        assert np.abs(g.sum(axis=1)).max() < 1e-14  # partition of unity


@pytest.mark.parametrize("npe", [4, 20])
def test_stress_oracle_reproduces_a_uniform_strain_field(npe):
    """Patch test: u = G x gives the strain sym(G) (engineering shear) at every node, stress = D strain."""
    from ferrix_b200 import decks
    from oracle import inp, stress
    text = decks.c3d4_cantilever(2, 2, 3) if npe == 4 else decks.c3d20_box(2, 2, 2)
    p = inp.parse_inp_text(text)
    xyz = np.asarray([p.nodes[i] for i in p.index_to_node_id])
    G = np.array([[1e-3, 2e-4, -3e-4], [5e-4, -2e-3, 1e-4], [-1e-4, 3e-4, 4e-4]])
    u = (xyz @ G.T).ravel()
    t = np.full(len(xyz), 20.0)
    S, E = stress.nodal_stress_strain(p, u, t, t)
    want = np.array([G[0, 0], G[1, 1], G[2, 2], G[0, 1] + G[1, 0], G[1, 2] + G[2, 1], G[0, 2] + G[2, 0]])
    assert np.abs(E - want).max() < 1e-12
    mat = p.materials[0]
    D = stress._d_matrix(mat.youngs_modulus.interpolate(20.0), mat.poisson_ratio.interpolate(20.0))
    assert np.abs(S - D @ want).max() < 1e-7 * np.abs(D @ want).max()


def test_mises_and_tresca_closed_forms():
    from oracle import stress
    S = np.array([[100.0, 0, 0, 0, 0, 0], [0, 0, 0, 50.0, 0, 0], [10.0, 10.0, 10.0, 0, 0, 0]])
    assert np.allclose(stress.mises(S), [100.0, np.sqrt(3.0) * 50.0, 0.0])
    assert np.allclose(stress.tresca(S), [100.0, 100.0, 0.0])
