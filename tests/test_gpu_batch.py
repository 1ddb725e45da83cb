"""Batched form: many molecules of uneven size in one set of launches, each
molecule's energy equal to the reference's (golden) and to its energy when
solved alone; molecules joining and leaving between iterations."""
import numpy as np
import pytest

from conftest import load_case
from dollarstorescf_b200.batch import Batch
from dollarstorescf_b200.engine import BOYS_REF

pytestmark = pytest.mark.gpu

MIX = ["water_sto3g", "water_631g", "ch4_631g", "c3h8_sto3g", "water_631gs", "dimer_631gs", "he_631g"]


def test_batch_energies_match_reference_and_alone():
    cases = [load_case(n) for n in MIX]
    with Batch(schwarz_threshold=0.0, boys_mode=BOYS_REF) as b:
        hs = [b.add(sh) for (_, _, sh) in cases]
        b.solve(conv=1e-10)
        mixed = [b.result(h)[0] for h in hs]
    for (d, _, _), E in zip(cases, mixed):
        assert abs(E - float(d["E"])) < 1e-9, (E, float(d["E"]))
    # alone
    for (d, _, sh), Em in zip(cases, mixed):
        with Batch(schwarz_threshold=0.0, boys_mode=BOYS_REF) as b:
            h = b.add(sh)
            b.solve(conv=1e-10)
            Ea = b.result(h)[0]
        assert abs(Ea - Em) < 1e-10


def test_batch_continuous_join_and_leave():
    d1, _, sh1 = load_case("water_631gs")
    d2, _, sh2 = load_case("ch4_631g")
    d3, _, sh3 = load_case("dimer_631gs")
    with Batch(schwarz_threshold=0.0, boys_mode=BOYS_REF) as b:
        h1 = b.add(sh1)
        h2 = b.add(sh2)
        b.step(3, conv=1e-10)          # both under way
        h3 = b.add(sh3)                # joins mid-flight
        done = {}
        for _ in range(200):
            act = b.step(1, conv=1e-10)
            for h in (h1, h2, h3):
                if h not in done and b.finished(h):
                    done[h] = b.result(h)[0]
                    b.remove(h)        # leaves; the others keep iterating
            if len(done) == 3:
                break
        assert len(done) == 3
    assert abs(done[h1] - float(d1["E"])) < 1e-9
    assert abs(done[h2] - float(d2["E"])) < 1e-9
    assert abs(done[h3] - float(d3["E"])) < 1e-9


def test_batch_pools_compact_under_churn():
    # Each admission appends the molecule's primitive pairs and work lists to
    # the batch's device pools; removals leave holes, and a pool that fills up
    # is compacted over the live molecules, moving their records.  Molecules
    # admitted first stay live while 300 others join and leave (several
    # compactions of both pools); their energies must still be the reference's.
    cases = [load_case(n) for n in MIX]
    _, _, churn = load_case("dimer_631gs")
    with Batch(schwarz_threshold=0.0, boys_mode=BOYS_REF) as b:
        hs = [b.add(sh) for (_, _, sh) in cases]
        b.step(2, conv=1e-10)
        for k in range(300):
            h = b.add(churn)
            if k % 50 == 0:
                b.step(1, conv=1e-10)  # the composition is rebuilt over the moved records
            b.remove(h)
        b.solve(conv=1e-10)
        out = [b.result(h)[0] for h in hs]
    for (d, _, _), E in zip(cases, out):
        assert abs(E - float(d["E"])) < 1e-9, (E, float(d["E"]))


def test_batch_admission_by_memory():
    d, _, sh = load_case("dimer_631gs")
    with Batch(arena_bytes=600_000) as b:   # one 36-function molecule needs about 0.33 MB: one fits, two do not
        b.add(sh)
        with pytest.raises(Exception) as e:
            b.add(sh)
        assert "not admitted" in str(e.value)


MIXED_SET = ["water_631gs", "dimer_631gs", "ch4_631g", "w4_631gs", "w8_631gs"]


def test_batch_mixed_form_within_one_microhartree_and_same_alone():
    """The incremental mixed-precision form run for a whole batch: every
    molecule within 1 uEh of the reference's energy, and its result the same
    when it is solved alone (its FP32/skip decisions depend on its own data only)."""
    cases = [load_case(n) for n in MIXED_SET]
    with Batch(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as b:
        hs = [b.add(sh) for (_, _, sh) in cases]
        b.solve(conv=1e-10, mixed=True)
        res = [b.result(h) for h in hs]
    for (d, _, _), (E, _, it, st) in zip(cases, res):
        assert st == 0
        assert abs(E - float(d["E"])) < 1e-6, (E, float(d["E"]))
    for (d, _, sh), (Em, _, itm, _) in zip(cases, res):
        with Batch(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as b:
            h = b.add(sh)
            b.solve(conv=1e-10, mixed=True)
            Ea, _, ita, st = b.result(h)
        assert st == 0
        assert abs(Ea - Em) < 1e-9, (Ea, Em)


def test_batch_switches_between_plain_and_mixed_forms():
    """A batch that runs a few mixed iterations and then finishes in the plain
    form ends at the plain form's energy (the switch forces a full build)."""
    d, _, sh = load_case("w4_631gs")
    with Batch(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as b:
        h = b.add(sh)
        b.step(5, conv=1e-10, mixed=True)
        b.solve(conv=1e-10)
        E, _, it, st = b.result(h)
    assert st == 0
    assert abs(E - float(d["E"])) < 1e-9


def test_batch_finished_poll_profile_and_tuner():
    """dss_batch_finished reports every molecule exactly once, in the step that
    produced its result; dss_batch_profile times the classes; the batch tuner's
    choice leaves the energies at the reference's."""
    from dollarstorescf_b200.autotune import tune_batch

    names = ["water_631gs", "dimer_631gs", "ch4_631g", "w4_631gs"]
    cases = [load_case(n) for n in names]
    with Batch(schwarz_threshold=1e-12, boys_mode=BOYS_REF) as b:
        hs = [b.add(sh) for (_, _, sh) in cases]
        ms = b.profile()
        assert sum(ms) > 0 and min(ms) >= 0
        assert tune_batch(b)
        seen = []
        for _ in range(200):
            b.step(1, conv=1e-10)
            seen += b.finished_handles()
            if len(seen) >= len(hs):
                break
        assert sorted(seen) == sorted(hs)
        for h, (d, _, _) in zip(hs, cases):
            E, _, it, st = b.result(h)
            assert st == 0
            assert abs(E - float(d["E"])) < 1e-9


def test_batch_persistent_launch_same_energies():
    # Persistent grouped launches (the L <= 2 and L = 3..4 thread-per-quartet
    # classes each in one kernel fed by a device work queue): the reference's
    # energies in the plain form, and the mixed form within 1 uEh of them.
    cases = [load_case(n) for n in MIX]
    for mixed, tol in ((False, 1e-9), (True, 1e-6)):
        with Batch(schwarz_threshold=0.0, boys_mode=BOYS_REF) as b:
            b.set_persistent(True)
            hs = [b.add(sh) for (_, _, sh) in cases]
            b.solve(conv=1e-10, mixed=mixed)
            for (d, _, _), h in zip(cases, hs):
                E, _, it, st = b.result(h)
                assert st == 0
                assert abs(E - float(d["E"])) < tol, (mixed, E, float(d["E"]))
            t = b.time_build()
            assert t > 0.0
