"""Serving: continuous batching of a seeded Poisson request stream.  Every
served energy equals the same molecule solved alone (the invariance the
serving form promises), displacements warm-started from the parent density
converge in fewer iterations, and latency statistics are reported."""
import numpy as np
import pytest

from dollarstorescf_b200 import geometry, serve
from dollarstorescf_b200.batch import Batch
from dollarstorescf_b200.engine import BOYS_REF

pytestmark = pytest.mark.gpu


def solo_energy(sh, guess=None):
    with Batch(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as b:
        h = b.add(sh, guess=guess)
        b.solve(conv=1e-10)
        return b.result(h)


def test_served_results_equal_solo_results():
    dimer = geometry.water_dimer(3)
    E0, D0 = serve.solve_parent(dimer)
    reqs = serve.make_request_stream(count=24, rate=200.0, seed=11, parent_density=D0, dimer=dimer)
    out = serve.serve(reqs, conv=1e-10)
    assert out["solves"] == len(reqs)
    assert out["p50_ms"] is not None and out["p99_ms"] >= out["p50_ms"]
    assert out["peak_inflight"] > 1  # requests overlapped on the device
    by_id = {r.rid: r for r in out["results"]}
    for req in reqs[:10]:
        res = by_id[req.rid]
        assert res.status == 0
        E, _, it, st = solo_energy(req.shells, req.guess)
        # |dE| between the mixed batch and the molecule alone: same kernels,
        # different launch composition, identical convergence path
        assert abs(res.energy - E) < 1e-9, (req.kind, res.energy, E)


def test_warm_start_from_parent_density():
    dimer = geometry.water_dimer(3)
    E0, D0 = serve.solve_parent(dimer)
    disp = geometry.displacements(dimer, 0.005)[5]
    from dollarstorescf_b200 import basis, shells
    sh = shells.build_shells(disp, basis.builtin_basis("6-31G*"), pure=True)
    Ew, _, itw, _ = solo_energy(sh, D0)
    Ec, _, itc, _ = solo_energy(sh, None)
    assert abs(Ew - Ec) < 1e-8
    assert itw < itc


def test_served_mixed_form_equals_solo_and_within_one_microhartree():
    """The mixed-precision incremental form served: each result equals the same
    molecule's mixed solve alone, and lies within 1 uEh of its FP64 energy."""
    dimer = geometry.water_dimer(3)
    E0, D0 = serve.solve_parent(dimer)
    reqs = serve.make_request_stream(count=16, rate=200.0, seed=5, parent_density=D0, dimer=dimer)
    out = serve.serve(reqs, conv=1e-10, mixed=True)
    assert out["solves"] == len(reqs)
    assert out["peak_inflight"] > 1
    by_id = {r.rid: r for r in out["results"]}
    for req in reqs[:8]:
        res = by_id[req.rid]
        assert res.status == 0
        with Batch(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as b:
            h = b.add(req.shells, guess=req.guess)
            b.solve(conv=1e-10, mixed=True)
            Em, _, _, _ = b.result(h)
        E64, _, _, _ = solo_energy(req.shells, req.guess)
        assert abs(res.energy - Em) < 1e-9, (req.kind, res.energy, Em)
        assert abs(res.energy - E64) < 1e-6, (req.kind, res.energy, E64)


def test_admission_waits_for_memory_and_results_do_not_change():
    """A small arena: the requests that do not fit wait until finished molecules
    free their regions (admissions_deferred > 0), and every result still equals
    the same molecule solved alone."""
    from dollarstorescf_b200 import basis, shells

    dimer = geometry.water_dimer(3)
    E0, D0 = serve.solve_parent(dimer)
    b631 = basis.builtin_basis("6-31G*")
    disps = geometry.displacements(dimer, 0.005)
    reqs = [serve.Request(i, 0.0, shells.build_shells(disps[i], b631, pure=True), "dimer displacement", guess=D0)
            for i in range(8)]
    with Batch(schwarz_threshold=1e-12, boys_mode=BOYS_REF, arena_bytes=1_000_000) as b:
        _, free_bytes, region = b.info(n_for_region=36)
        fits = free_bytes // region
        assert 1 <= fits < len(reqs)
        out = serve.serve(reqs, conv=1e-10, batch=b)
    assert out["solves"] == len(reqs) and out["converged"] == len(reqs)
    assert out["admissions_deferred"] > 0
    assert out["peak_inflight"] <= fits
    assert out["queue_p99_ms"] > 0.0
    for req, res in zip(reqs, sorted(out["results"], key=lambda r: r.rid)):
        E, _, it, st = solo_energy(req.shells, req.guess)
        assert abs(res.energy - E) < 1e-9, (res.rid, res.energy, E)


def test_pipelined_serving_results_equal_solo_results():
    # Two batches, each with its own context, stream and host thread, overlap
    # on the GPU: every request is still answered, each energy equals the same
    # molecule solved alone, and both batches carried work.
    dimer = geometry.water_dimer(3)
    E0, D0 = serve.solve_parent(dimer)
    reqs = serve.make_request_stream(count=24, rate=200.0, seed=11, parent_density=D0, dimer=dimer)
    out = serve.serve_pipelined(reqs, pipelines=2, conv=1e-10)
    assert out["solves"] == len(reqs) and out["converged"] == len(reqs)
    assert out["pipelines"] == 2 and out["peak_inflight"] > 1
    by_id = {r.rid: r for r in out["results"]}
    assert sorted(by_id) == sorted(r.rid for r in reqs)
    for req in reqs[:8]:
        res = by_id[req.rid]
        E, _, it, st = solo_energy(req.shells, req.guess)
        assert abs(res.energy - E) < 1e-9, (req.kind, res.energy, E)
