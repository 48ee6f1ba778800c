"""Groups (bnm_group_*): subjects of different node counts, each with its own
SC, targets and autotuned integrator, run one generation as one CUDA graph.
The eager first call, and the graph launches after it, must give the same
results as each plan's own bnm_run on the same inputs."""
import numpy as np
import pytest

import bnm_cuda_b200 as B
from bnm_cuda_b200 import synth

pytestmark = pytest.mark.gpu

NODES = (16, 48, 160)  # register kernel, register kernel, cluster kernel


def _subjects(n):
    plans, params = [], []
    for k, N in enumerate(NODES):
        sc = synth.make_sc(N, 0.3, 10 + k)
        cfg = B.Config(nodes=N, max_sims=8, time_steps=12000, bold_tr=500, window_size=10, window_step=2,
                       bold_remove_s=2)
        s = cfg.sizes()
        rng = np.random.default_rng(k)
        plans.append(B.Plan(cfg, sc, rng.uniform(-0.2, 0.8, s["n_pairs"]), rng.uniform(-0.3, 1.0, 300)))
        params.append(synth.uniform_params(n, N, 30 + k))
    return plans, params


def _same(a, b):
    np.testing.assert_array_equal(a["fic_ntrials"], b["fic_ntrials"])
    np.testing.assert_array_equal(a["fic_failed"], b["fic_failed"])
    for k in ("cost", "fic_penalty", "fc_corr", "fc_diff", "fcd_ks"):
        np.testing.assert_allclose(a[k], b[k], rtol=0, atol=1e-9, err_msg=k)
    np.testing.assert_allclose(a["w_ie"], b["w_ie"], rtol=0, atol=1e-9)


def test_group_graph_matches_per_plan_runs():
    plans, params = _subjects(5)
    solo = [p.run(*prm, outputs=("w_ie",)) for p, prm in zip(plans, params)]
    with B.Group(plans) as g:
        first = g.run(params)
        assert not g.last()["graph"]
        second = g.run(params)
        assert g.last()["graph"] and g.last()["ms"] > 0
        for a, b, c in zip(solo, first, second):
            _same(a, b)
            _same(a, c)
        # new parameters, same batch sizes: the graph is reused
        params2 = [synth.uniform_params(5, p.cfg.nodes, 99 + k) for k, p in enumerate(plans)]
        third = g.run(params2)
        assert g.last()["graph"]
    for p, prm, r in zip(plans, params2, third):
        _same(p.run(*prm, outputs=("w_ie",)), r)
    kinds = [p.integrator()["kind"] for p in plans]
    assert kinds == ["register", "register", "cluster"], kinds
    for p in plans:
        p.close()


def test_group_tunes_fresh_plans_for_sm_time():
    """Plans first run through a group are tuned by SM time (the launch's time
    weighted by the fraction of the GPU it fills), and keep that shape: a later
    bnm_run of the same batch size gives the group's results exactly."""
    plans, params = _subjects(6)
    with B.Group(plans) as g:
        first = g.run(params)
        second = g.run(params)
        for a, b in zip(first, second):
            _same(a, b)
    kinds = [p.integrator()["kind"] for p in plans]
    assert kinds[:2] == ["register", "register"], kinds
    assert kinds[2] in ("cluster", "colsplit", "colsplit2"), kinds
    assert all(p.integrator()["tried"] >= 2 for p in plans)
    for p, prm, r in zip(plans, params, first):
        _same(p.run(*prm, outputs=("w_ie",)), r)
    for p in plans:
        p.close()


def test_group_rejects_bad_inputs():
    plans, params = _subjects(3)
    with B.Group(plans) as g:
        bad = list(params)
        G = bad[1][0].copy()
        G[0] = np.inf
        bad[1] = (G, bad[1][1], bad[1][2])
        with pytest.raises(B.BnmError) as e:
            g.run(bad)
        assert e.value.code == B.BNM_EINVAL
        with pytest.raises(B.BnmError):
            g.run([(np.ones(9), 0.2, 0.2)] + params[1:])  # more than max_sims
        g.run(params)  # still usable
    with pytest.raises(B.BnmError):
        B.Group([plans[0], plans[0]])
    for p in plans:
        p.close()


@pytest.mark.parametrize("N", [48, 160])
def test_single_plan_generation_is_one_graph_launch(N, monkeypatch):
    """bnm_run: the first call for a batch size runs eagerly (and tunes the
    integrator); later calls with device FIC are one graph launch of the whole
    generation.  The graph must give the eager path's results (same tuned
    shape, same stream operations), with and without the optional BOLD / FC /
    FCD outputs, for new parameters as well, and its stage timings must be
    valid."""
    sc = synth.make_sc(N, 0.3, 3)
    cfg = B.Config(nodes=N, max_sims=6, time_steps=12000, bold_tr=500, window_size=10, window_step=2,
                   bold_remove_s=2)
    s = cfg.sizes()
    rng = np.random.default_rng(1)
    emp_fc, emp_fcd = rng.uniform(-0.2, 0.8, s["n_pairs"]), rng.uniform(-0.3, 1.0, 300)
    P1, P2 = synth.uniform_params(6, N, 40), synth.uniform_params(6, N, 41)
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        e1 = p.run(*P1)
        assert not p.graph_launched()
        g1 = p.run(*P1, outputs=("w_ie",))
        assert p.graph_launched()
        _same(e1, g1)
        g2 = p.run(*P2)  # full outputs through the graph
        assert p.graph_launched()
        t = p.timings()
        assert t["integrate"] > 0 and t["total"] >= t["integrate"]
        monkeypatch.setenv("BNM_B200_GRAPH", "0")
        e2 = p.run(*P2)
        assert not p.graph_launched()
    _same(e2, g2)
    for k in ("bold", "fc", "fcd", "ext_means"):
        np.testing.assert_array_equal(e2[k], g2[k], err_msg=k)


@pytest.mark.parametrize("n", [200, 400])  # fewer / more particles than the 296 resident CTAs
def test_particle_placement_keeps_every_particles_result(n, monkeypatch):
    """Particle placement (on by default for the register kernel): the CTAs
    take particles in an order predicted from the plan's history (heaviest
    FIC work on the CTAs alone on an SM, the lightest on the second CTA of an
    SM).  Placement changes only where a particle runs, so every particle's
    results must equal those of the unplaced plan (BNM_B200_PLACE=0), bit for
    bit, with more particles than SMs (paired and lone CTAs), with more
    particles than resident CTAs (CTAs claim again from both ends until the
    claims meet) and on the graph path."""
    N = 20
    sc = synth.make_sc(N, 0.3, 6)
    cfg = B.Config(nodes=N, max_sims=n, time_steps=12000, bold_tr=500, window_size=10, window_step=2,
                   bold_remove_s=2)
    s = cfg.sizes()
    rng = np.random.default_rng(2)
    emp_fc, emp_fcd = rng.uniform(-0.2, 0.8, s["n_pairs"]), rng.uniform(-0.3, 1.0, 300)
    P1, P2 = synth.uniform_params(n, N, 50), synth.uniform_params(n, N, 51)
    monkeypatch.setenv("BNM_B200_SLOTS", "1")
    monkeypatch.setenv("BNM_B200_PLACE", "0")
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        assert p.placement() == dict(enabled=False, placed_last=False)
        ref = [p.run(*P1), p.run(*P2)]
    monkeypatch.delenv("BNM_B200_PLACE")
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        got = [p.run(*P1)]  # no history yet: identity order
        assert p.placement() == dict(enabled=True, placed_last=False)
        monkeypatch.setenv("BNM_B200_GRAPH", "0")
        got.append(p.run(*P2))  # placed, eager
        assert not p.graph_launched() and p.placement()["placed_last"]
        monkeypatch.delenv("BNM_B200_GRAPH")
        got.append(p.run(*P2))  # placed, graph launch
        assert p.graph_launched() and p.placement()["placed_last"]
    for a, b in ((ref[0], got[0]), (ref[1], got[1]), (ref[1], got[2])):
        _same(a, b)
        np.testing.assert_array_equal(a["cost"], b["cost"])


def test_group_places_its_own_batch_after_a_larger_run(monkeypatch):
    """A plan whose last bnm_run placed a larger batch (an order over 40
    particles) then runs 12 particles in a group, eagerly and as a graph: the
    group sets the order for its own batch, so every particle is simulated
    and the results equal an unplaced plan's."""
    N = 20
    sc = synth.make_sc(N, 0.3, 6)
    cfg = B.Config(nodes=N, max_sims=40, time_steps=12000, bold_tr=500, window_size=10, window_step=2,
                   bold_remove_s=2)
    s = cfg.sizes()
    rng = np.random.default_rng(3)
    emp_fc, emp_fcd = rng.uniform(-0.2, 0.8, s["n_pairs"]), rng.uniform(-0.3, 1.0, 300)
    big, small = synth.uniform_params(40, N, 60), synth.uniform_params(12, N, 61)
    monkeypatch.setenv("BNM_B200_SLOTS", "1")
    monkeypatch.setenv("BNM_B200_PLACE", "0")
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as q:
        want = q.run(*small, outputs=("w_ie",))
    monkeypatch.delenv("BNM_B200_PLACE")
    p = B.Plan(cfg, sc, emp_fc, emp_fcd)
    p.run(*big)
    p.run(*big)
    assert p.placement()["placed_last"]
    with B.Group([p]) as g:
        for _ in range(2):  # eager (tunes for 12), then the graph
            _same(want, g.run([small])[0])
        assert g.last()["graph"]
    p.close()


def test_cluster_pairing_by_predicted_work_keeps_every_particles_result(monkeypatch):
    """Two-particle column-split clusters (N = 200) with placement: after the
    first batch a cluster advances two particles of similar predicted FIC
    work instead of two neighbours by index.  A particle's results do not
    depend on its partner (a restart the partner asks for reruns it bit for
    bit), so they must equal the unplaced plan's, eagerly and as a graph."""
    N, n = 200, 16  # one batch of 16 is the history placement needs
    sc = synth.make_sc(N, 0.3, 7)
    cfg = B.Config(nodes=N, max_sims=n, time_steps=12000, bold_tr=500, window_size=10, window_step=2,
                   bold_remove_s=2)
    s = cfg.sizes()
    rng = np.random.default_rng(4)
    emp_fc, emp_fcd = rng.uniform(-0.2, 0.8, s["n_pairs"]), rng.uniform(-0.3, 1.0, 300)
    P1, P2 = synth.uniform_params(n, N, 70), synth.uniform_params(n, N, 71)
    monkeypatch.setenv("BNM_B200_SHAPE", "4,25,4,2,25")
    monkeypatch.setenv("BNM_B200_PLACE", "0")
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        ref = p.run(*P2, outputs=("bold", "w_ie"))
    monkeypatch.delenv("BNM_B200_PLACE")
    with B.Plan(cfg, sc, emp_fc, emp_fcd) as p:
        p.run(*P1)
        assert p.placement() == dict(enabled=True, placed_last=False)
        monkeypatch.setenv("BNM_B200_GRAPH", "0")
        got = [p.run(*P2, outputs=("bold", "w_ie"))]  # placed, eager
        assert p.placement()["placed_last"] and not p.graph_launched()
        monkeypatch.delenv("BNM_B200_GRAPH")
        got.append(p.run(*P2, outputs=("bold", "w_ie")))  # placed, graph launch
        assert p.graph_launched()
        assert p.integrator()["kind"] == "colsplit2"
    for g in got:
        _same(ref, g)
        np.testing.assert_array_equal(ref["cost"], g["cost"])
        np.testing.assert_array_equal(ref["bold"], g["bold"])
