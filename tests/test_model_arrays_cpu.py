"""fx_model_from_arrays (the binary mesh path) builds the same model as the deck
parser, checked on the host without a GPU: node index order, coordinates, element
groups and connectivity, material tables, step descriptions and their load / BC
records (src/solver/parser.rs:111-482, src/solver/mesh_lib/mesh.rs:35-50)."""
import gzip
import os

import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks
from tests.deck_arrays import arrays_from_deck


def _deck(golden_dir, name):
    with gzip.open(os.path.join(golden_dir, "decks", name + ".inp.gz"), "rt") as fh:
        return fh.read()


def _same_model(a, b):
    assert (a.num_nodes, a.num_elements, len(a.steps), a.num_materials) == \
        (b.num_nodes, b.num_elements, len(b.steps), b.num_materials)
    assert np.array_equal(a.mesh.index_to_node_id, b.mesh.index_to_node_id)
    xa, ga = a.export()
    xb, gb = b.export()
    assert np.array_equal(xa, xb)
    for npe in (4, 20):
        assert np.array_equal(ga[npe][0], gb[npe][0]) and np.array_equal(ga[npe][1], gb[npe][1])
    for sa, sb in zip(a.steps, b.steps):
        assert (sa.info.nlgeom, sa.info.solver, sa.info.increment) == (sb.info.nlgeom, sb.info.solver,
                                                                       sb.info.increment)
        for is_bc in (False, True):
            for ra, rb in zip(sa.records(is_bc), sb.records(is_bc)):
                assert np.array_equal(ra, rb)


@pytest.mark.parametrize("name", ["C3D4_staticstep", "C3D4_2staticstep", "C3D20", "NLGEOM_test"])
def test_arrays_match_parser_on_reference_decks(golden_dir, name):
    text = _deck(golden_dir, name)
    _same_model(fx.Project.from_inp_text(text), fx.Project.from_arrays(**arrays_from_deck(text)))


@pytest.mark.parametrize("make", [lambda: decks.c3d4_nlgeom_beam(6, 2, 2),          # E(T), *EXPANSION, amplitude
                                  lambda: decks.c3d20_box(2, 3, 4),
                                  lambda: decks.c3d4_cantilever(3, 3, 5)])
def test_arrays_match_parser_on_synthetic_decks(make):
    text = make()
    _same_model(fx.Project.from_inp_text(text), fx.Project.from_arrays(**arrays_from_deck(text)))


def test_arrays_reject_inconsistent_descriptions():
    kw = arrays_from_deck(decks.c3d4_cantilever(1, 1, 1))
    bad_dof = dict(kw, steps=[dict(kw["steps"][0], loads=[(1, 3, 1.0, -1, 1)])])
    bad_amp = dict(kw, steps=[dict(kw["steps"][0], loads=[(1, 0, 1.0, 5, 1)])])
    ids, conn, mat = kw["c3d4"]
    bad_mat = dict(kw, c3d4=(ids, conn, np.full_like(mat, 7)))
    for bad, what in ((bad_dof, "dof"), (bad_amp, "amplitude"), (bad_mat, "material")):
        with pytest.raises(fx.FerrixError) as e:
            fx.Project.from_arrays(**bad)
        assert e.value.kind == "InvalidArgument" and what in e.value.message, e.value.message


def test_arrays_later_node_definition_wins():
    """A repeated node id keeps the later coordinates, as a deck that defines a node twice."""
    kw = arrays_from_deck(decks.c3d4_cantilever(1, 1, 1))
    ids = np.concatenate([kw["node_ids"], kw["node_ids"][:1]])
    xyz = np.concatenate([kw["xyz"], kw["xyz"][:1] + 5.0])
    p = fx.Project.from_arrays(**dict(kw, node_ids=ids, xyz=xyz))
    x, _ = p.export()
    k = int(np.searchsorted(p.mesh.index_to_node_id, kw["node_ids"][0]))
    assert np.array_equal(x[k], kw["xyz"][0] + 5.0) and p.num_nodes == len(kw["node_ids"])


@pytest.mark.parametrize("spec", [lambda: decks.c3d4_cantilever_spec(2, 2, 3), lambda: decks.c3d20_box_spec(2, 2, 3),
                                  lambda: decks.c3d4_nlgeom_beam_spec(6, 2, 2)])
def test_generator_arrays_match_its_deck_text(spec):
    """decks.deck_arrays(spec) (no text) gives the model that parsing write_deck(spec) gives."""
    s = spec()
    _same_model(fx.Project.from_inp_text(decks.write_deck(s)), fx.Project.from_arrays(**decks.deck_arrays(s)))


def test_population_arrays_match_population_decks():
    texts = decks.batch_population(6, seed=3, c3d20_fraction=0.5)
    arrs = decks.batch_population(6, seed=3, c3d20_fraction=0.5, arrays=True)
    for (t, d1), (a, d2) in zip(texts, arrs):
        assert d1 == d2
        _same_model(fx.Project.from_inp_text(t), fx.Project.from_arrays(**a))
