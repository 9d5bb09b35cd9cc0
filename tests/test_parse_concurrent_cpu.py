"""The .inp parser from several host threads at once (request-loop slots parse their decks
concurrently; the parser's parallel loops share one pool of worker threads): every
concurrent parse gives the same mesh arrays as a parse alone, and a deck with an error
still reports it. Host-only: fx_model_from_inp without a context, no GPU needed."""
import ctypes as C
import threading

import numpy as np
import pytest

import ferrix_b200 as fx
from ferrix_b200 import decks


def _parse_export(lib, text: bytes):
    h = C.c_void_p()
    rc = lib.fx_model_from_inp(None, text, len(text), C.byref(h))
    if rc != 0:
        return rc, None
    n4, n20 = C.c_int64(), C.c_int64()
    assert lib.fx_model_export(h, None, C.byref(n4), None, None, C.byref(n20), None, None) == 0
    nn, ne, ns, nm = C.c_int64(), C.c_int64(), C.c_int(), C.c_int()
    assert lib.fx_model_sizes(h, C.byref(nn), C.byref(ne), C.byref(ns), C.byref(nm)) == 0
    xyz = np.empty(3 * nn.value)
    c4 = np.empty(4 * n4.value, dtype=np.int32)
    m4 = np.empty(n4.value, dtype=np.int32)
    c20 = np.empty(20 * n20.value, dtype=np.int32)
    m20 = np.empty(n20.value, dtype=np.int32)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    assert lib.fx_model_export(h, p(xyz), C.byref(n4), p(c4), p(m4), C.byref(n20), p(c20), p(m20)) == 0
    lib.fx_model_destroy(h)
    return 0, (xyz, c4, m4, c20, m20)


def test_concurrent_parses_match_a_parse_alone():
    lib = fx._lib.load()
    texts = [decks.c3d20_box(6, 6, 24).encode(), decks.c3d4_cantilever(6, 6, 20).encode(),
             decks.c3d20_box(4, 5, 9, seed=3).encode()]
    bad = texts[1].replace(b"*Node\n1, 0.0, 0.0, 0.0", b"*Node\n1, 0.0, abc, 0.0", 1)  # a node line that does not parse
    assert bad != texts[1]
    alone = [_parse_export(lib, t) for t in texts]
    rc_bad, _ = _parse_export(lib, bad)
    assert rc_bad != 0 and all(rc == 0 for rc, _ in alone)
    results = {}

    def worker(k):
        out = []
        for r in range(3):
            i = (k + r) % (len(texts) + 1)
            out.append((i, _parse_export(lib, texts[i] if i < len(texts) else bad)))
        results[k] = out

    th = [threading.Thread(target=worker, args=(k,)) for k in range(6)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert len(results) == 6
    for out in results.values():
        for i, (rc, arrays) in out:
            if i == len(texts):
                assert rc == rc_bad
                continue
            assert rc == 0
            for a, b in zip(arrays, alone[i][1]):
                assert np.array_equal(a, b)


@pytest.mark.filterwarnings("ignore:This process .* is multi-threaded:DeprecationWarning")
def test_parse_in_a_forked_child():
    """A child forked after the parser's workers started (they are not copied by fork, and
    the queue's lock may be held) parses on its own thread and gets the same arrays."""
    import os
    import select
    import signal
    lib = fx._lib.load()
    text = decks.c3d20_box(6, 6, 24).encode()
    rc, alone = _parse_export(lib, text)  # starts the workers in this process
    assert rc == 0
    r, w = os.pipe()
    pid = os.fork()
    if pid == 0:  # child: parse, report, leave without running the parent's cleanup
        ok = 0
        try:
            rc2, arrays = _parse_export(lib, text)
            ok = int(rc2 == 0 and all(np.array_equal(a, b) for a, b in zip(arrays, alone)))
        finally:
            os.write(w, bytes([ok]))
            os._exit(0)
    os.close(w)
    ready, _, _ = select.select([r], [], [], 60.0)  # a child stuck on an inherited lock is ended
    got = os.read(r, 1) if ready else b""
    os.close(r)
    if not ready:
        os.kill(pid, signal.SIGKILL)
    os.waitpid(pid, 0)
    assert got == b"\x01"
