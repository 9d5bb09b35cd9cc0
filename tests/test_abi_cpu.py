"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and its `.inp` parser builds the same model as the oracle's
restatement of src/solver/parser.rs (no compute call is made)."""
import ctypes as C
import gzip
import os

import numpy as np
import pytest

from ferrix_b200 import _lib, decks
import ferrix_b200 as fx
from oracle import inp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ferrix_b200.h")


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    declared = _lib.header_symbols(HEADER)
    assert len(declared) >= 20
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    assert set(declared) == set(_lib.SIGNATURES), set(declared) ^ set(_lib.SIGNATURES)


def _struct_fill_check(struct_type, fill_fn):
    """fill_fn writes exactly sizeof(struct_type) bytes: a guard region after the
    ctypes struct (sized from the Python field list) stays untouched, so the
    Python layout is at least as long as the C one."""
    import ctypes as C
    n = C.sizeof(struct_type)
    buf = (C.c_ubyte * (n + 64))(*([0xA5] * (n + 64)))
    fill_fn(C.cast(buf, C.POINTER(struct_type)))
    assert bytes(buf[n:]) == b"\xa5" * 64
    return struct_type.from_buffer_copy(bytes(buf[:n]))


def test_option_structs_match_the_header():
    lib = _lib.load()
    o = _struct_fill_check(_lib.SolveOpts, lib.fx_default_solve_opts)
    assert o.precision == fx.PREC_MIXED and o.preconditioner == fx.PRECOND_AMG and o.rtol == 1e-8
    assert o.amg_smoother_degree == 2 and o.amg_overcorrect == 0.0 and o.amg_cheb_ratio == 0.0
    so = _struct_fill_check(_lib.ServerOpts, lib.fx_default_server_opts)
    assert so.slots == 4 and so.opts.amg_aggregate_nodes == 40 and so.opts.amg_cheb_ratio == 0.0
    # the last field of each struct as the header lists it
    text = open(HEADER).read()
    body = text[text.index("typedef struct {", text.index("fx_precision;")):text.index("} fx_solve_opts;")]
    import re
    body = re.sub(r"/\*.*?\*/", "", body[body.index("{") + 1:], flags=re.S)
    names = [d.split()[-1] for d in body.split(";") if d.strip()]
    assert names == [f[0] for f in _lib.SolveOpts._fields_], names


def _compare(text):
    o = inp.parse_inp_text(text)
    m = inp.model_arrays(o) if o.nodes else None
    p = fx.Project.from_inp_text(text)
    assert p.num_nodes == len(o.nodes)
    assert p.num_elements == len(o.elements)
    assert len(p.steps) == len(o.steps)
    assert p.num_materials == len(o.materials)
    if m is not None:
        assert np.array_equal(p.mesh.index_to_node_id, m.node_ids)
        xyz, groups = p.export()
        assert np.array_equal(xyz, m.xyz, equal_nan=True)
        for npe in (4, 20):
            conn, mat = groups[npe]
            if npe in m.groups:
                assert np.array_equal(conn, m.groups[npe][1]) and np.array_equal(mat, m.groups[npe][2])
            else:
                assert conn.size == 0
    for k, (ps, os_) in enumerate(zip(p.steps, o.steps)):
        assert ps.info.nlgeom == os_.nlgeom and ps.info.solver == os_.solver
        inc = os_.increment
        assert ps.info.increment == (inc.initial_time_increment, inc.time_period, inc.min_time_increment,
                                     inc.max_time_increment)
        for is_bc, recs in ((False, os_.loads), (True, os_.bcs)):
            ids, dofs, vals, org, tab = ps.records(is_bc)
            assert len(ids) == len(recs)
            for i, r in enumerate(recs):
                assert (ids[i], dofs[i], vals[i], org[i], bool(tab[i])) == \
                    (r.node_id, r.dof, r.value, r.origin_step, r.amplitude.times is not None)
    return p, o


@pytest.mark.parametrize("name", ["C3D4_staticstep", "C3D4_2staticstep", "C3D20", "NLGEOM_test"])
def test_parser_matches_oracle_on_reference_decks(golden_dir, name):
    with gzip.open(os.path.join(golden_dir, "decks", name + ".inp.gz"), "rt") as fh:
        _compare(fh.read())


def test_parser_matches_oracle_on_synthetic_decks():
    _compare(decks.c3d4_cantilever(2, 2, 4))
    _compare(decks.c3d20_box(2, 2, 3))
    _compare(decks.c3d4_nlgeom_beam(4, 2, 2))


def _relabel(text, node_id, elem_id, seed):
    """The same deck with node / element ids mapped through node_id / elem_id, the
    *NODE and *ELEMENT lines shuffled, one node and one element defined twice (the
    later definition must win) and the volume elset assigned a material twice."""
    rng = np.random.default_rng(seed)
    out, block, kw = [], [], None

    def flush():
        if kw in ("NODE", "ELEMENT") and block:
            order = rng.permutation(len(block))
            rows = [block[i] for i in order]
            first = rows[0].split(",")
            if kw == "NODE":  # redefine a node: moved by 1e-3 in x
                rows.append(", ".join([first[0], repr(float(first[1]) + 1e-3)] + first[2:]))
            else:  # redefine an element with its nodes rotated (C3D4: 1, 2, 3, 4 -> 1, 3, 4, 2)
                f = [x.strip() for x in first]
                rows.append(", ".join(f[:2] + f[3:5] + [f[2]] + f[5:]))
            out.extend(rows)
        else:
            out.extend(block)
        block.clear()

    for line in text.splitlines():
        if line.startswith("*"):
            flush()
            kw = line[1:].split(",")[0].strip().upper() if not line.startswith("**") else kw
            out.append(line)
            if line.upper().startswith("*SOLID SECTION"):
                out.append(line)
            continue
        f = [x.strip() for x in line.split(",")]
        if kw == "NODE":
            f[0] = str(node_id(int(f[0])))
        elif kw == "ELEMENT":
            f = [str(elem_id(int(f[0])))] + [str(node_id(int(x))) for x in f[1:] if x]
        elif kw == "NSET":
            f = [str(node_id(int(x))) if x.isdigit() else x for x in f if x]
        elif kw == "ELSET":
            f = [str(elem_id(int(x))) if x.isdigit() else x for x in f if x]
        block.append(", ".join(f))
    flush()
    return "\n".join(out) + "\n"


@pytest.mark.parametrize("node_id,elem_id", [
    (lambda i: i, lambda e: e),                      # consecutive ids, shuffled lines
    (lambda i: 3 * i + 5, lambda e: 2 * e + 1),      # gaps: direct table
    (lambda i: 100003 * i, lambda e: 7919 * e),      # sparse: hash map
], ids=["consecutive", "gaps", "sparse"])
def test_parser_id_layouts_match_oracle(node_id, elem_id):
    """Bulk *NODE / *ELEMENT blocks (over 1,024 lines) with shuffled, gapped and
    repeated ids parse to the oracle's arrays (nodes by ascending id, later
    definitions winning)."""
    text = _relabel(decks.c3d4_cantilever(8, 8, 40), node_id, elem_id, seed=3)
    p, o = _compare(text)
    assert p.num_nodes == 9 * 9 * 41 and p.num_elements == 8 * 8 * 40 * 6


def test_preprocess_chunks_match_oracle():
    """A deck of several MB (the preprocessor splits it into chunks on several
    threads) with a solver name to substitute at its very end."""
    text = decks.c3d20_box(14, 14, 30)
    assert len(text) > 2 << 20
    text = text.replace("*Static, Solver=Spooles", "*Static, Solver=Iterative Cholesky")
    text = text.replace("*Element", "*Heading\nPardiso, Spooles, Iterative Cholesky Scaling\n*Element", 1)
    p, o = _compare(text)
    assert p.steps[0].info.solver == "ITERATIVE"


def _reformat(text, seed):
    """The same deck with the formatting the preprocessor must undo: CRLF line ends,
    random letter case, spaces and tabs around fields, comment and blank lines
    between data lines, and data lines split after a comma (continuation lines)."""
    rng = np.random.default_rng(seed)
    out = []
    for line in text.split("\n"):
        if rng.random() < 0.05:
            out.append("** c" + ("," if rng.random() < 0.5 else ""))  # comment lines never continue
        if rng.random() < 0.03:
            out.append(" \t ")
        if not line.startswith("**") and rng.random() < 0.5:
            line = "".join(ch.lower() if rng.random() < 0.5 else ch for ch in line)
        if "," in line and not line.startswith("*") and rng.random() < 0.3:
            k = line.index(",")  # split after the first comma
            head, tail = line[:k + 1], line[k + 1:]
            out.append("  " + head + " \t")
            line = tail
        out.append(("\t" if rng.random() < 0.1 else "") + line + (" " if rng.random() < 0.2 else ""))
    return "\r\n".join(out)


@pytest.mark.parametrize("seed", [1, 2])
def test_parser_formatting_matches_oracle(seed):
    """Multi-chunk decks (over 2 MB, so the preprocessor runs several threads) with CRLF,
    mixed case, whitespace, interleaved comments / blank lines and continuation lines."""
    text = _reformat(decks.c3d20_box(14, 14, 30), seed)
    assert len(text) > 2 << 20
    p, o = _compare(text)
    assert p.num_nodes == len(o.nodes) > 0


EDGE_DECKS = {
    "empty": "",
    "comments_only": "** a\n**b,\n   \n",
    # line-by-line path (blocks under 1,024 lines): a later definition of a node / element wins
    "repeated_ids": "*NODE\n1,0,0,0\n2,1,0,0\n1,5,5,5\n3,0,1,0\n4,0,0,1\n*ELEMENT,TYPE=C3D4,ELSET=E\n"
                    "1,1,2,3,4\n1,2,1,3,4\n",
    "element_without_type": "*NODE\n1,0,0,0\n*ELEMENT\n1,1,1,1,1\n",  # data dropped
    "plus_sign_and_exponents": "*NODE\n+1,1E3,-2.5e-2,+3.\n2,inf,0,0\n",
    # f64::from_str forms beside plain decimals: NaN / infinity spellings, out-of-range
    # magnitudes (to inf and to zero), a bare fraction or integer part, a negative zero
    "float_forms": "*NODE\n1,.5,5.,-0\n2,1e999,-1e-400,NaN\n3,infinity,-Inf,1E+05\n4,-.25e1,+0.0,7\n",
    # the same forms in a block of 1,100 lines (the bulk parse of *NODE data)
    "float_forms_bulk": "*NODE\n" + "".join(
        "%d,%s,%s,%s\n" % (i + 1, ("0.1", ".5", "1e999", "NaN", "-Inf", "+2.5")[i % 6],
                             ("5.", "-1e-400", "3", "-0", "1E+05", "infinity")[i % 6], repr(i * 0.37))
        for i in range(1100)),
}


@pytest.mark.parametrize("name", list(EDGE_DECKS))
def test_parser_edge_decks_match_oracle(name):
    _compare(EDGE_DECKS[name])


QUIRKS = """** comment
*Heading
title line
*Node
1, 0, 0, 0
2, 1.0, 0, 0
3, 0, 1.0, 0
4, 0, 0, 1.0
5, 1E0, 1e0, +1.0
*Element, type=C3D4, elset=E1
1, 1, 2, 3, 4
2, 2, 3, 4,
5
*Nset, nset=ALL
1, 2, 3,
4, 5
*Elset, elset=E2
E1
*Material, name=Steel
*Elastic
210000, 0.3, 20
190000, 0.3, 300
*Expansion, zero=20
1.2e-5
*Solid section, elset=E2, material=STEEL
*Amplitude, name=A1, shiftx=0.5
0, 0, 1, 2
*Initial conditions, type=temperature
ALL, 50
3, 70
*Boundary
1, 1, 3
2, 4, 6
*Step, nlgeom, inc=50
*Static, solver=pardiso
0.25, 1.0, 1e-4, 0.5
*Boundary, op=new
1, 1, 3, 0.0
2, 2
*Cload, amplitude=A1
ALL, 2, 10.0
5, 3, -1.5
*Node print, nset=ALL
U
*Cload
4, 1, 99.0
*End step
*Step
*Static, Solver=Iterative Scaling
*Cload, op=NEW
3, 3, 2.5
*Dload
*End step
"""


def test_parser_quirks_match_oracle():
    p, o = _compare(QUIRKS)
    assert p.steps[0].info.nlgeom and p.steps[0].info.solver == "DIRECT"
    assert p.steps[1].info.solver == "ITERATIVE"
    assert o.initial_temperatures[3] == 70.0


@pytest.mark.parametrize("text,kind", [
    ("*ORIENTATION, NAME=X\n", "UnsupportedKeyword"),
    ("*STEP\n*STATIC, SOLVER=MAGIC\n", "UnknownSolver"),
    # one substitution pass: ITERATIVE CHOLESKY -> ITERATIVE leaves "ITERATIVE SCALING", not replaced again
    ("*STEP\n*STATIC, SOLVER=ITERATIVE CHOLESKY SCALING\n", "UnknownSolver"),
    ("*NODE\n1, 0, 0\n", "ParseError"),
    ("*MATERIAL\n", "ParseError"),
    ("*SOLID SECTION, MATERIAL=M\n", "ParseError"),
    ("*SOLID SECTION, ELSET=A, MATERIAL=M\n", "MaterialNotFound"),
    ("*MATERIAL, NAME=M\n*SOLID SECTION, ELSET=A, MATERIAL=M\n", "ElsetNotFound"),
    ("*MATERIAL, NAME=M\n*SOLID SECTION, ELSET=A, MATERIAL=Q\n", "MaterialNotFound"),
    ("*ELEMENT, TYPE=C3D8\n1, 1, 2, 3, 4, 5, 6, 7, 8\n", "ParseError"),
    ("*ELEMENT, TYPE=C3D4\n1, 1, 2, 3\n", "ParseError"),
    ("*NODE\n1, 0, 0, 0, 7\n", "ParseError"),
    ("*NODE\n1, 0, x, 0\n", "ParseError"),
    ("*NODE\n-1, 0, 0, 0\n", "ParseError"),
    ("*AMPLITUDE\n0, 1\n", "ParseError"),
])
def test_parser_errors(text, kind):
    with pytest.raises(inp.FerrixError) as eo:
        inp.parse_inp_text(text)
    assert eo.value.kind == kind
    with pytest.raises(fx.FerrixError) as eg:
        fx.Project.from_inp_text(text)
    assert eg.value.kind == kind
    # the variant's payload crosses the C ABI (fx_last_error_detail): the deck line of
    # ParseError / UnsupportedKeyword, the keyword, material / set / solver name or message
    e, o = eg.value, eo.value
    assert e.text == o.message, (e.text, o.message)
    if kind in ("ParseError", "UnsupportedKeyword"):
        assert e.line == o.line, (e.line, o.line)
    else:
        assert e.line is None
    assert e.id is None


def test_error_detail_without_context_is_per_thread():
    """fx_last_error_detail(NULL) reports the calling thread's last failure."""
    import threading
    lib = _lib.load()
    seen = {}

    def parse(tag, text):
        with pytest.raises(fx.FerrixError):
            fx.Project.from_inp_text(text)
        d = _lib.ErrorDetail()
        assert lib.fx_last_error_detail(None, C.byref(d)) == 0
        seen[tag] = (d.status, d.line, d.text.decode())

    t = threading.Thread(target=parse, args=("other", "*NODE\n1, 0, 0, 0\n*FOO\n"))
    t.start()
    t.join()
    parse("main", "*STEP\n*STATIC, SOLVER=MAGIC\n")
    assert seen["other"] == (4, 3, "FOO")
    assert seen["main"] == (5, -1, "MAGIC")
