"""results.vtk.series, the ParaView time series of the reference's VtkWriter
(src/solver/io/vtk.rs:46-70 init, :305-318 one entry per written increment,
:325-333 finish): the C-ABI writers reproduce its bytes, including the comma after
the last entry and Rust's `{}` display of an f64 (shortest round-trip decimal, never
in exponent form). Host-only: no GPU needed."""
import os

import ferrix_b200 as fx

HEADER = '{\n          "file-series-version" : "1.0",\n          "files" : [\n'
FOOTER = "  ]\n}\n"


def _series(lib, d, entries):
    assert lib.fx_vtk_series_init(os.fsencode(d)) == 0
    for name, t in entries:
        assert lib.fx_vtk_series_add(os.fsencode(d), name.encode(), t) == 0
    assert lib.fx_vtk_series_finish(os.fsencode(d)) == 0
    with open(os.path.join(d, "results.vtk.series")) as fh:
        return fh.read()


def test_series_bytes_match_the_reference(tmp_path):
    lib = fx._lib.load()
    d = str(tmp_path / "job" / "Job-1")  # created with its parents, as create_dir_all does
    text = _series(lib, d, [("step_1_1.vtk", 0.1), ("step_1_2.vtk", 0.30000000000000004),
                            ("step_1_3.vtk", 1.0), ("step_2_1.vtk", 1e-05), ("step_2_2.vtk", 12.5)])
    assert text == (HEADER
                    + '{ "name" : "step_1_1.vtk", "time" : 0.1 },\n'
                    + '{ "name" : "step_1_2.vtk", "time" : 0.30000000000000004 },\n'
                    + '{ "name" : "step_1_3.vtk", "time" : 1 },\n'
                    + '{ "name" : "step_2_1.vtk", "time" : 0.00001 },\n'
                    + '{ "name" : "step_2_2.vtk", "time" : 12.5 },\n'
                    + FOOTER)


def test_init_starts_a_new_series(tmp_path):
    lib = fx._lib.load()
    d = str(tmp_path)
    _series(lib, d, [("a.vtk", 1.0)])
    assert _series(lib, d, []) == HEADER + FOOTER


def test_unwritable_directory_is_a_generic_io_error(tmp_path):
    lib = fx._lib.load()
    blocker = tmp_path / "file"
    blocker.write_text("x")
    d = os.fsencode(str(blocker / "sub"))  # a directory below a regular file cannot exist
    assert fx._lib.STATUS_NAMES[lib.fx_vtk_series_init(d)] == "GenericIo"
    assert lib.fx_vtk_series_add(d, b"x.vtk", 1.0) != 0
    assert lib.fx_vtk_series_finish(None) != 0
