"""Host-side logic: loaders, geometry generators, packed layout, shells."""
import os

import numpy as np
import pytest

from dollarstorescf_b200 import basis, geometry, shells

SAMPLE = """\
! comment
H     0
S    3   1.00
      0.1873113696D+02       0.3349460434D-01
      0.2825394365D+01       0.2347269535D+00
      0.6401216923D+00       0.8137573261D+00
S    1   1.00
      0.1612777588D+00       1.0000000
****
C     0
S    1   1.00
      0.3047524880D+01       1.0
SP   2   1.00
      0.2324918408D+01      -0.3509174574D-01       0.8941508043D-02
      0.6324303556D+00      -0.1912328431D+00       0.1410094640D+00
D    1   1.00
      0.8000000000D+00       1.0000000
****
"""


def test_parse_basis_sp_split_and_d_exponents():
    bs = basis.parse_basis_text(SAMPLE)
    assert [s.l for s in bs.elements[1]] == [0, 0]
    assert bs.elements[1][0].exps[0] == pytest.approx(18.73113696)
    c = bs.elements[6]
    assert [s.l for s in c] == [0, 0, 1, 2]
    assert c[1].exps == c[2].exps
    assert c[2].coefs[1] == pytest.approx(0.1410094640)


def test_parse_basis_errors():
    with pytest.raises(basis.BasisError, match="recognized angular momentum"):
        basis.parse_basis_text("H 0\nQ 1 1.0\n 1.0 1.0\n****\n")
    with pytest.raises(basis.BasisError, match="range of 1-100"):
        basis.parse_basis_text("H 0\nS 0 1.0\n****\n")
    with pytest.raises(basis.BasisError, match="positive exponents"):
        basis.parse_basis_text("H 0\nS 1 1.0\n -1.0 1.0\n****\n")
    with pytest.raises(basis.BasisError, match="could not be found"):
        basis.read_basis("/nonexistent/basis")


def test_builtin_bases_shell_structure():
    b = basis.builtin_basis("6-31G*")
    assert [(s.l, len(s.exps)) for s in b.elements[8]] == [(0, 6), (0, 3), (1, 3), (0, 1), (1, 1), (2, 1)]
    assert [(s.l, len(s.exps)) for s in b.elements[1]] == [(0, 3), (0, 1)]
    assert [(s.l, len(s.exps)) for s in basis.builtin_basis("STO-3G").elements[6]] == [(0, 3), (0, 3), (1, 3)]
    with pytest.raises(basis.BasisError):
        basis.builtin_basis("cc-pVQZ")


def test_read_xyz(tmp_path):
    p = tmp_path / "w.xyz"
    p.write_text("3\n\nO 0 0 0\nH 0.7576 0.5870 0\nH -0.7576 0.5870 0\n")
    m = basis.read_xyz(str(p))
    assert m.Z == [8, 1, 1]
    assert m.xyz[1][0] == pytest.approx(0.7576 * 1.889726126)
    bad = tmp_path / "b.xyz"
    bad.write_text("2\n\nO 0 0 0\n")
    with pytest.raises(basis.GeometryError, match="atoms expected"):
        basis.read_xyz(str(bad))
    bad.write_text("1\n\nXx 0 0 0\n")
    with pytest.raises(basis.GeometryError, match="not a valid element"):
        basis.read_xyz(str(bad))


def test_basis_function_counts():
    w = geometry.water_cluster(3, 3, 2, 16, 0)
    b = basis.builtin_basis("6-31G*")
    assert shells.build_shells(w, b, pure=True).nbf() == 288
    assert shells.build_shells(w, b, pure=False).nbf() == 304
    assert shells.build_shells(w, b, pure=False).nshell == 160
    w32 = geometry.water_cluster(4, 4, 2, 32, 0)
    assert shells.build_shells(w32, b, pure=False).nbf() == 608
    assert shells.build_shells(geometry.water(), basis.builtin_basis("STO-3G")).nbf() == 7


def test_water_cluster_is_seeded_and_physical():
    a = geometry.water_cluster(3, 3, 2, 16, 5)
    b = geometry.water_cluster(3, 3, 2, 16, 5)
    assert a.xyz == b.xyz
    X = np.array(a.xyz) / basis.A_TO_BOHR
    Z = np.array(a.Z)
    d = np.linalg.norm(X[:, None] - X[None], axis=-1)
    np.fill_diagonal(d, 99)
    assert d.min() > 0.9  # no clashes
    oh = d[np.ix_(Z == 8, Z == 1)].min(axis=0)
    assert np.allclose(oh, 0.9572, atol=1e-3)


@pytest.mark.parametrize("n", [1, 2, 5, 10])
def test_alkane_generator(n):
    m = geometry.alkane(n, 0, jitter=0.0)
    Z = np.array(m.Z)
    assert (Z == 6).sum() == n and (Z == 1).sum() == 2 * n + 2
    X = np.array(m.xyz) / basis.A_TO_BOHR
    d = np.linalg.norm(X[:, None] - X[None], axis=-1)
    ch = d[np.ix_(Z == 1, Z == 6)].min(axis=1)
    assert np.allclose(ch, 1.09, atol=1e-6)
    if n > 1:
        cc = np.sort(d[np.ix_(Z == 6, Z == 6)], axis=1)[:, 1]
        assert np.allclose(cc, 1.54, atol=1e-6)


def test_displacements():
    m = geometry.water_dimer(0)
    ds = geometry.displacements(m, 0.005)
    assert len(ds) == 36
    delta = np.array(ds[0].xyz) - np.array(m.xyz)
    assert delta[0, 0] == pytest.approx(0.005) and np.count_nonzero(delta) == 1


def test_packed_layout_roundtrip():
    rng = np.random.default_rng(0)
    A = rng.standard_normal((7, 7))
    A = A + A.T
    p = shells.pack(A)
    # element (y <= x) at x(x+1)/2 + y
    assert p[shells.packed_index(2, 5)] == A[2, 5]
    assert p[5 * 6 // 2 + 2] == A[2, 5]
    assert np.array_equal(shells.unpack(p, 7), A)


def _replica_worker(rank, world, port, out):
    import os

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench

    # Each replica reports its own time; the job's time is the slowest one.
    t = bench.max_over_ranks(1.0 + rank, "cpu")
    out.put((rank, t, bench.replica_rate(world, 10, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_bench_replicas_take_the_slowest_rank_gloo():
    """bench.py --gpus N runs N independent replicas (the Fock build does not
    shard here): every rank gets the maximum time, and the whole-job rate is
    N x steps over it.  Two gloo ranks on the CPU."""
    import random

    import torch.multiprocessing as mp

    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = random.randint(20000, 40000)
    procs = [ctx.Process(target=_replica_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [2.0, 2.0]
    assert all(abs(r[2] - 10.0) < 1e-12 for r in res)


def test_whole_build_refinement_finds_the_concurrent_optimum():
    # refine_whole: coordinate descent over per-class shapes on a whole-build
    # time.  A fake build whose time depends on the joint choice (class "a"
    # is best with shape 1 only when "b" runs shape 0, as concurrency can make
    # it) must end at the joint minimum, keep the starting shape of a class
    # whose alternatives are rejected, and report both times.
    from dollarstorescf_b200.autotune import refine_whole

    state = {0: 0, 1: 5, 2: 0}

    def set_variant(i, v):
        if i == 2 and v != 0:
            raise ValueError("shape not available for this class")
        state[i] = v

    def time_build():
        t = 10.0
        t -= 2.0 if (state[0] == 1 and state[1] == 0) else 0.0
        t -= 1.0 if state[1] == 0 else 0.0
        return t

    choice = {"a": 0, "b": 5, "c": 0}
    classes = [(1, "b", (0, 5)), (0, "a", (0, 1)), (2, "c", (0, 1))]
    out = refine_whole(time_build, set_variant, classes, choice, repeats=1)
    assert choice == {"a": 1, "b": 0, "c": 0}
    assert state == {0: 1, 1: 0, 2: 0}
    assert out["ms_whole_build_per_class_choice"] == 10.0 and out["ms_whole_build"] == 7.0


@pytest.mark.parametrize("case", ["c4_631g", "c7_631g", "c10_631g", "c6_631gs", "w16_631gs", "w16_631gs_6d"])
def test_newton_schulz_overlap_inverse_root_converges_in_32_iterations(case):
    # The batch computes X = S^-1/2 of new molecules by 32 coupled Newton-Schulz
    # iterations (Y0 = S/c, Z0 = I, T = (3I - ZY)/2, Y <- YT, Z <- TZ, X = Z/sqrt(c),
    # c = the largest absolute row sum) and accepts X when max |X S X - I| <= 1e-11,
    # else falls back to the eigen-decomposition.  The same arithmetic in numpy on
    # the reference's own overlap matrices (alkanes of the batched form, the bench's
    # water cluster) must pass that check and agree with U s^-1/2 U^T.
    d = np.load(os.path.join(os.path.dirname(__file__), "golden", case + ".npz"))
    n = int(d["nbf"])
    S = d["S"] if d["S"].ndim == 2 else shells.unpack(d["S"], n)
    c = np.abs(S).sum(axis=1).max()
    Y, Z = S / c, np.eye(n)
    for _ in range(32):
        T = 1.5 * np.eye(n) - 0.5 * Z @ Y
        Y, Z = Y @ T, T @ Z
    X = Z / np.sqrt(c)
    assert np.abs(X @ S @ X - np.eye(n)).max() <= 1e-11
    w, U = np.linalg.eigh(S)
    assert np.abs(X - (U / np.sqrt(w)) @ U.T).max() < 1e-9
