"""GPU tests of the continuous-batching server: each request's rows are the
same when it is served in a mix as when it is searched alone (byte for byte
on the popcount path, where the ring's slices join in genome order), and
arrivals join the requests already on the GPU at the next slice boundary."""
import random
import threading
import time

import pytest

import randgen

pytestmark = pytest.mark.gpu


def _genome_and_requests(cof_mod, seed=31, n_req=12):
    rng = random.Random(seed)
    _, records = randgen.random_genome(rng, 3, 20000, 40000)
    reqs = []
    for k in range(n_req):
        filt, mk, mm = randgen.REQUEST_SHAPES[k % len(randgen.REQUEST_SHAPES)]
        guides = ["".join(rng.choice("ACGT") for _ in range(25)) for _ in range(rng.randint(1, 6))]
        pats = [mk(x) for x in guides]
        for p in pats:
            randgen.plant_sites(rng, records, p, filt, 3, 2)
        db, rb = ((1, 1) if k % 4 == 3 else (0, 0))
        reqs.append(dict(search_filter=filt, patterns=pats, max_mismatches=min(mm, 3),
                         max_dna_bulges=db, max_rna_bulges=rb))
    g = cof_mod.Genome()
    for name, data, _nibs, s, e in randgen.chunk_records(rng, records, 4000):
        g.add_chunk(name, data, s, e)
    return g, reqs


@pytest.mark.parametrize("per_pass,ring", [(0, 0), (1, 0), (0, 1), (0, 7)])
def test_server_matches_alone(cof_mod, per_pass, ring):
    g, reqs = _genome_and_requests(cof_mod)
    alone = [g.search(**r) for r in reqs]
    srv = cof_mod.Server(g, max_requests_per_pass=per_pass, ring_slices=ring)
    tickets = [srv.submit(**r) for r in reqs]
    got = [srv.wait(t) for t in tickets]
    st = srv.stats()
    srv.close()
    for r, (text, n, lat), (ref, nref) in zip(reqs, got, alone):
        if r["max_dna_bulges"] or r["max_rna_bulges"]:
            assert sorted(text.splitlines()) == sorted(ref.splitlines())
        else:
            assert text == ref  # slices joined in genome order: the same text
        assert n == nref
        assert lat > 0
    assert st["completed"] == len(reqs)
    if per_pass == 1:
        assert st["passes"] == len(reqs) and st["largest_pass"] == 1
    else:
        assert st["largest_pass"] > 1
        if ring == 7:  # every request takes one full turn of 7 slices
            assert st["passes"] >= 7
        else:
            assert st["passes"] < len(reqs)


def test_arrival_joins_the_ring_mid_turn(cof_mod):
    # a request submitted while another is on the ring joins it at the next
    # slice boundary: the two share steps, so the ring takes fewer steps
    # than two turns, and both results equal their own searches
    rng = random.Random(41)
    _, records = randgen.random_genome(rng, 4, 400000, 600000)
    reqs = []
    for k in range(2):
        filt, mk, mm = randgen.REQUEST_SHAPES[k]
        pats = [mk("".join(rng.choice("ACGT") for _ in range(25))) for _ in range(40)]
        for p in pats[:4]:
            randgen.plant_sites(rng, records, p, filt, 5, 2)
        reqs.append(dict(search_filter=filt, patterns=pats, max_mismatches=3))
    g = cof_mod.Genome()
    for name, data, _nibs, s, e in randgen.chunk_records(rng, records, 60000):
        g.add_chunk(name, data, s, e)
    alone = [g.search(**r) for r in reqs]
    k = 16
    srv = cof_mod.Server(g, ring_slices=k)
    t0 = srv.submit(**reqs[0])
    deadline = time.time() + 60
    while srv.stats()["passes"] < 2 and time.time() < deadline:
        pass
    st_mid = srv.stats()
    t1 = srv.submit(**reqs[1])
    got = [srv.wait(t0), srv.wait(t1)]
    st = srv.stats()
    srv.close()
    assert 2 <= st_mid["passes"] < k and st_mid["completed"] == 0
    assert st["largest_pass"] == 2 and st["passes"] < 2 * k
    for (text, n, _lat), (ref, nref) in zip(got, alone):
        assert text == ref and n == nref


def test_server_concurrent_submitters(cof_mod):
    g, reqs = _genome_and_requests(cof_mod, seed=32, n_req=16)
    alone = [g.search(**r) for r in reqs]
    srv = cof_mod.Server(g)
    out = [None] * len(reqs)

    def client(i):
        t = srv.submit(**reqs[i])
        out[i] = srv.wait(t)

    th = [threading.Thread(target=client, args=(i,)) for i in range(len(reqs))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    srv.close()
    for (text, n, _lat), (ref, nref) in zip(out, alone):
        assert sorted(text.splitlines()) == sorted(ref.splitlines()) and n == nref


def test_server_bad_ticket_and_timeout(cof_mod):
    g, reqs = _genome_and_requests(cof_mod, seed=33, n_req=2)
    srv = cof_mod.Server(g)
    with pytest.raises(cof_mod.CofError) as e:
        srv.wait(999)
    assert e.value.code == cof_mod.COF_E_BADINPUT
    t = srv.submit(**reqs[0])
    try:
        srv.wait(t, timeout_ms=0)
    except cof_mod.CofError as ex:  # still pending: bounded wait gives up
        assert ex.code == cof_mod.COF_E_TIMEOUT
        srv.wait(t)
    srv.close()
