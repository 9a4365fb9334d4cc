"""Serving loop (ffb_server_*): requests admitted by memory budget into
concurrent slots and traced in slices, round-robin; each result equals the
same solve run alone, and the traces of different requests interleave on the
device."""
import numpy as np
import pytest

from form_factors_b200 import native, scenes

pytestmark = pytest.mark.gpu


def _requests():
    return [(scenes.parallel_plates(6, 1.0), 800, 21), (scenes.icosphere(3, 1.0, inward=True), 300, 22),
            (scenes.clutter(150, 0.08, seed=2, enclosure_cells=4), 500, 23), (scenes.unit_box(), 5000, 24),
            (scenes.perpendicular_plates(8), 600, 25), (scenes.icosphere(2, 0.7, inward=True), 900, 26)]


def test_results_in_the_mix_equal_results_alone(ctx):
    reqs = _requests()
    server = native.Server(0, budget_bytes=0, slots=3)
    ids = [server.submit(f, rpf, seed) for f, rpf, seed in reqs]
    infos = [server.wait(i, timeout_s=300) for i in ids]
    assert all(inf.state == 2 for inf in infos)
    for (f, rpf, seed), rid in zip(reqs, ids):
        got = server.result(rid, len(f))
        ctx.scene_set(f)
        ctx.grid_build(cells_per_face=32)
        want = ctx.form_factor_counts(np.full(len(f), rpf, np.int32), np.zeros(len(f), np.int32), seed=seed, epoch=0)
        assert np.array_equal(got, want)
        server.release(rid)
    st = server.stats()
    assert 1 <= st.peak_running <= 3  # never more than the slots
    assert st.reserved_bytes == 0 and st.queued == 0 and st.running == 0
    server.close()


def test_admission_by_memory_budget():
    reqs = _requests()
    n_max = max(len(f) for f, _, _ in reqs)
    # room for the largest request alone (4 N^2 + 1536 N + 8 MiB), not for two
    budget = 4 * n_max * n_max + 1536 * n_max + (8 << 20) + (1 << 20)
    server = native.Server(0, budget_bytes=budget, slots=4)
    ids = [server.submit(f, rpf, seed) for f, rpf, seed in reqs]
    # a finished result keeps its reservation until released: a client that
    # consumes results in order lets the next request in
    for i in ids:
        assert server.wait(i, timeout_s=120).state == 2
        assert server.stats().reserved_bytes <= budget
        server.release(i)
    # the largest request fills the budget: at most two of the small ones fit together
    assert 1 <= server.stats().peak_running <= 2
    # a request larger than the whole budget is refused at submit
    big = scenes.icosphere(5, 1.0)  # 20480 faces: 1.7 GB of counts
    with pytest.raises(native.FFBError) as e:
        server.submit(big, 10, 1)
    assert e.value.code == -305
    assert server.stats().reserved_bytes == 0
    server.close()


def test_traces_of_requests_overlap_on_the_device(ctx):
    """Two requests of 20 480 faces x 3000 rays (four 16 Mi-ray slices each)
    submitted together: their traces interleave on the device -- each
    request's span, from its first trace block's start to its last warp's end
    (%globaltimer, stamped by the kernel itself), overlaps the other's -- and
    each result equals the same solve run alone."""
    faces = scenes.icosphere(5, 1.0, inward=True)
    n = len(faces)
    server = native.Server(0, budget_bytes=0, slots=2)
    server.set_slicing(16 << 20, 2)
    ids = [server.submit(faces, 3000, seed) for seed in (41, 42)]
    infos = [server.wait(i, timeout_s=300) for i in ids]
    assert all(inf.state == 2 for inf in infos)
    assert all(inf.slices == 4 for inf in infos), [inf.slices for inf in infos]
    (a0, a1), (b0, b1) = [(inf.trace_start_ns, inf.trace_end_ns) for inf in infos]
    assert 0 < a0 < a1 and 0 < b0 < b1
    assert max(a0, b0) < min(a1, b1), "device spans do not overlap: %s" % ([(a0, a1), (b0, b1)],)
    assert server.stats().peak_tracing == 2
    ctx.scene_set(faces)
    ctx.grid_build(cells_per_face=32)
    for rid, seed in zip(ids, (41, 42)):
        want = ctx.form_factor_counts(np.full(n, 3000, np.int32), np.zeros(n, np.int32), seed=seed, epoch=0)
        assert np.array_equal(server.result(rid, n), want)
        server.release(rid)
    server.close()


def test_shortest_first_admission_and_its_age_limit(ctx):
    """One slot; a large request, a second large one, then two small ones.
    Shortest-first admits the small ones before the second large request;
    with an age limit of zero the oldest request always goes first, which is
    arrival order.  Results are those of the same solve alone."""
    big = scenes.icosphere(4, 1.0, inward=True)  # 5 120 faces
    small = scenes.parallel_plates(4, 1.0)       # 32 faces
    for shortest, limit in ((True, 600.0), (True, 0.0), (False, 0.0)):
        server = native.Server(0, budget_bytes=0, slots=1)
        server.set_admission(shortest_first=shortest, max_wait_s=limit)
        ids = [server.submit(big, 2000, 1), server.submit(big, 2000, 2), server.submit(small, 100, 3),
               server.submit(small, 100, 4)]
        # collected in completion order (ffb_server_wait_any)
        order, infos_by = [], {}
        pending = list(ids)
        while pending:
            rid, inf = server.wait_any(pending, timeout_s=300)
            order.append(rid)
            infos_by[rid] = inf
            pending.remove(rid)
        infos = [infos_by[i] for i in ids]
        assert all(inf.state == 2 for inf in infos)
        q = [inf.queue_s for inf in infos]
        if shortest and limit > 0:
            assert order.index(ids[2]) < order.index(ids[1]) and order.index(ids[3]) < order.index(ids[1]), order
        else:
            assert order == ids, order
        if shortest and limit > 0:
            assert q[2] < q[1] and q[3] < q[1], q  # the small requests overtake the second large one
        else:
            assert q[1] < q[2] < q[3], q           # arrival order
        got = server.result(ids[2], len(small))
        ctx.scene_set(small)
        ctx.grid_build(cells_per_face=32)
        want = ctx.form_factor_counts(np.full(len(small), 100, np.int32), np.zeros(len(small), np.int32), seed=3,
                                      epoch=0)
        assert np.array_equal(got, want)
        for i in ids:
            server.release(i)
        server.close()
