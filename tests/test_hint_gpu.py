"""The offline hint's ring multiply on the device (alto_hint_ring; YServer::answer_hint_ring, src/server.rs:656-768)
over the engine's resident database, against the oracle's schoolbook negacyclic products on sampled columns: at the
scheme's ring dimension (n = 2048) on a 1 GiB database and at a smaller ring, with and without the output
permutation.  The reference's own hint depends on spiral-rs's pseudorandom query and cannot be run here, so the query
polynomials are seeded uniform values mod Q (parity with the reference unpinned; the formula is pinned by
tests/test_oracle.py)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

Q = 4294955009


@pytest.mark.parametrize("rows,record_bytes,n,perm_out", [(32768, 32768, 2048, False), (4096, 4096, 256, True),
                                                        (2048, 8192, 2048, True)])
def test_hint_ring_matches_oracle(gpu, svc, eng, oracle, rows, record_bytes, n, perm_out):
    p = svc.Params(rows, record_bytes, n=n)
    st = svc.SyntheticState.make(p, seed=111)
    e = eng.Engine.from_state(st)
    rng = np.random.default_rng(112)
    query = rng.integers(0, Q, (rows // n, n), dtype=np.uint64)
    got = e.hint_ring(query, perm_out=perm_out)
    assert got.shape == (n, record_bytes) and (got < Q).all()
    for c0 in sorted(set(int(x) for x in rng.integers(0, record_bytes - 4, 3))) + [record_bytes - 4]:
        want = oracle.hint_ring(st.db_col, query, n, c0, c0 + 4, perm_out)
        assert np.array_equal(got[:, c0:c0 + 4], want), c0
    # the same engine, once more: the call keeps no state between calls
    assert np.array_equal(e.hint_ring(query, perm_out=perm_out), got)
    e.close()
