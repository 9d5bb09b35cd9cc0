"""Per-increment results (ResultWriter::write_increment, src/solver/step/static_step.rs:219-248)
on the GPU: Step.solve hands every converged increment to the writer with the reference's
step id, increment counter and global time, and the model holds that increment's
displacements while the writer runs. Compared with the oracle's Newton run of the same deck,
increment by increment (same ids and times; displacements within 1e-8 in the 2-norm), and
VtkWriter's files and results.vtk.series checked on disk.
"""
import os

import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks
from oracle import inp, static_step

pytestmark = pytest.mark.gpu

TOL_NLGEOM = 1e-8
DECK = dict(nx=12, ny=3, nz=3, tip_load=2.0e3, increments=4)


def _rust_f64(t: float) -> str:
    """Rust's `{}` of an f64: shortest round-trip digits, never in exponent form."""
    r = repr(float(t))
    if "e" in r or "E" in r:
        from decimal import Decimal
        r = format(Decimal(r), "f")
    return r[:-2] if r.endswith(".0") else r


@pytest.fixture(scope="module")
def beam():
    text = decks.c3d4_nlgeom_beam(**DECK)
    seen = []
    o = inp.parse_inp_text(text)
    o.default_initial_temperature = 20.0
    static_step.Runner(o, on_increment=lambda s, i, t, u: seen.append((s, i, t, u))).run()
    ctx = fx.Context(0)
    p = fx.Project.from_inp_text(text, ctx)
    p.default_initial_temperature = 20.0
    yield p, seen
    p.close()
    ctx.close()


def test_writer_sees_every_converged_increment(beam):
    p, ref = beam
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)
    got = []

    class Recorder:
        def write_increment(self, inc, timer):
            view = fx.SolutionState(p.num_dofs, p.num_nodes)
            view.project = inc.project
            got.append((inc.step_id, inc.inc_id, inc.time, view.displacements))

    p.steps[0].solve(1, p, st, writer=Recorder())
    assert [(s, i) for s, i, _, _ in got] == [(s, i) for s, i, _, _ in ref]
    assert len(got) == DECK["increments"]
    for (_, i, t, u), (_, _, t_ref, u_ref) in zip(got, ref):
        assert t == t_ref, (i, t, t_ref)
        err = float(np.linalg.norm(u - u_ref) / np.linalg.norm(u_ref))
        assert err <= TOL_NLGEOM, (i, err)
    assert np.array_equal(got[-1][3], st.displacements)  # the last increment is the step's result


def test_vtk_writer_files_and_series(beam, tmp_path):
    p, ref = beam
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)
    d = str(tmp_path / "Job-1")
    w = fx.VtkWriter(p, d)
    w.init()
    p.steps[0].solve(1, p, st, writer=w)
    w.finish()
    names = [f"step_{s}_{i}.vtk" for s, i, _, _ in ref]
    for n in names:
        with open(os.path.join(d, n)) as fh:
            assert fh.readline().startswith("# vtk DataFile Version 3.0")
    with open(os.path.join(d, "results.vtk.series")) as fh:
        text = fh.read()
    want = '{\n          "file-series-version" : "1.0",\n          "files" : [\n'
    for n, (_, _, t, _) in zip(names, ref):
        want += '{ "name" : "%s", "time" : %s },\n' % (n, _rust_f64(t))
    assert text == want + "  ]\n}\n"


def test_writer_error_ends_the_step(beam):
    p, _ = beam
    st = fx.SolutionState(p.num_dofs, p.num_nodes)
    st.initialize(p)

    class Failing:
        calls = 0

        def write_increment(self, inc, timer):
            Failing.calls += 1
            if inc.inc_id == 2:
                raise OSError("disk full")

    with pytest.raises(OSError):
        p.steps[0].solve(1, p, st, writer=Failing())
    assert Failing.calls == 2  # the step stopped at the failing increment
