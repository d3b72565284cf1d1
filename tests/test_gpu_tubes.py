"""Batched tubes in one persistent launch against the oracle's per-tube run
(the reference's rk_step on a ny = 1 grid, pinned by tests/golden/tubes.npz).

The FP64-exact launch reproduces every tube bit for bit; each tube's result
does not depend on its batch mates (a dt per tube); the CUDA-graph replay
equals the eager launch; the mixed form stays within 1e-5 density L1.
"""
import numpy as np
import pytest
import torch

from helpers import bitwise_equal, max_rel
from oracle import oracle

from hlld_ai_b200.tubes import TubeBatch, TubeStates, random_tubes, tube_prims

pytestmark = pytest.mark.gpu
G = 5.0 / 3.0


def small_batch(n=6, seed=7, lmin=32, lmax=96):
    return random_tubes(n, seed=seed, lmin=lmin, lmax=lmax, gamma=G)


def oracle_tube(states, i, ng, tend, limiter="weno5z", solver="hlld", max_steps=1 << 30):
    p = tube_prims(states, i, ng)
    L = int(states.lengths[i])
    t, steps = oracle.tube_run(p, L, ng, 1.0 / L, 0.4, tend, limiter, solver, G, max_steps=max_steps)
    return p, t, steps


@pytest.mark.parametrize("limiter", ["weno5z", "mc", "mp5"])
def test_exact_tubes_bitwise_oracle(limiter):
    st = small_batch()
    b = TubeBatch(st, limiter=limiter, precision="fp64_exact")
    b.launch(tend=0.03)
    torch.cuda.synchronize()
    for i in range(b.n):
        p, t, steps = oracle_tube(st, i, b.ng, 0.03, limiter)
        assert int(b.steps_out[i]) == steps
        assert float(b.t_out[i]) == t
        got = b.tube(i)
        for k in p:
            assert bitwise_equal(got[k], p[k]), (i, k, max_rel(p[k], got[k]))


def test_fp64_tubes_close_to_oracle():
    st = small_batch(seed=11)
    b = TubeBatch(st, limiter="weno5z", precision="fp64")
    b.launch(tend=0.05)
    torch.cuda.synchronize()
    for i in range(b.n):
        p, t, steps = oracle_tube(st, i, b.ng, 0.05)
        got = b.tube(i)
        for k in ("rho", "p", "vx", "By"):
            assert max_rel(p[k], got[k]) < 1e-8, (i, k)


def test_tube_result_independent_of_batch():
    st = small_batch(n=5, seed=3)
    whole = TubeBatch(st, precision="fp64_exact")
    whole.launch(tend=0.03)
    one = TubeStates(st.lengths[2:3], {k: v[2:3] for k, v in st.left.items()},
                     {k: v[2:3] for k, v in st.right.items()}, st.Bx[2:3])
    alone = TubeBatch(one, precision="fp64_exact")
    alone.launch(tend=0.03)
    torch.cuda.synchronize()
    a, b = whole.tube(2), alone.tube(0)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_graph_replay_equals_eager():
    st = small_batch(n=8, seed=5)
    eager = TubeBatch(st, precision="fp64")
    eager.launch(tend=0.02)
    graphed = TubeBatch(st, precision="fp64")
    g = graphed.capture(tend=0.02)
    graphed.reset()
    g.replay()
    torch.cuda.synchronize()
    for i in range(st.lengths.size):
        a, b = eager.tube(i), graphed.tube(i)
        for k in a:
            assert np.array_equal(a[k], b[k]), (i, k)
    assert torch.equal(eager.steps_out, graphed.steps_out)


def test_mixed_tubes_density_l1():
    st = small_batch(n=8, seed=9, lmin=128, lmax=256)
    ref = TubeBatch(st, precision="fp64")
    mix = TubeBatch(st, precision="mixed")
    ref.launch(tend=0.05)
    mix.launch(tend=0.05)
    torch.cuda.synchronize()
    for i in range(st.lengths.size):
        a, b = ref.tube(i)["rho"], mix.tube(i)["rho"]
        assert np.abs(a - b).mean() <= 1e-5, i


def test_autotune_picks_a_shape():
    st = small_batch(n=16, seed=13)
    b = TubeBatch(st, precision="fp64")
    threads, blocks = b.autotune(tend=0.005, sample=16)
    assert threads in (64, 128, 256) and blocks > 0
    b.launch(tend=0.01)
    torch.cuda.synchronize()
    assert bool((b.t_out > 0).all())
