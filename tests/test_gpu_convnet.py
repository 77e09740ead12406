"""Learned-correction network: forward and backward kernels (CUDA-core and
tcgen05) against the torch-CPU oracle, and training on PM-generated pairs."""
import numpy as np
import pytest

from oracle import convnet_ref as CR

pytestmark = pytest.mark.gpu


def _net(n, seed=3):
    from cola_halo_b200.learned import ConvNet
    net = ConvNet(n, seed)
    # non-trivial biases and a larger output layer than the initialisation
    p = net.params()
    rng = np.random.default_rng(seed)
    for l in range(3):
        b0 = l * CR.LAYER + CR.WSZ
        p[b0: b0 + (16 if l < 2 else 3)] = rng.normal(0, 0.1, 16 if l < 2 else 3)
    w2 = 2 * CR.LAYER
    p[w2: w2 + CR.WSZ] *= 10
    net.set_params(p)
    return net, p


def _inputs(n, seed=5):
    rng = np.random.default_rng(seed)
    return rng.normal(0, 1, (n, n, n, 2)).astype(np.float32)


def test_forward_simt_matches_oracle(gpu_lib):
    n = 32
    net, p = _net(n)
    net.tensor_cores(False)
    x = _inputs(n)
    got = net.forward_host(x)
    want = CR.forward(x, p)[0].detach().numpy()
    err = np.abs(got - want).max() / np.abs(want).max()
    assert err < 1e-2, err          # bf16 hidden activations round at different points
    assert np.corrcoef(got.ravel(), want.ravel())[0, 1] > 0.9999


def test_backward_matches_oracle(gpu_lib):
    n = 32
    net, p = _net(n)
    net.tensor_cores(False)
    x = _inputs(n)
    g3 = np.random.default_rng(8).normal(0, 1, (n, n, n, 3)).astype(np.float32)
    got = net.backward_host(x, g3)
    want = CR.grads(x, p, g3)
    live = want != 0
    cos = np.dot(got[live], want[live]) / np.linalg.norm(got[live]) / np.linalg.norm(want[live])
    rel = np.linalg.norm(got[live] - want[live]) / np.linalg.norm(want[live])
    assert cos > 0.9999 and rel < 2e-2, (cos, rel)
    # masked weights (unused channels) get no gradient to speak of
    assert np.abs(got[~live]).max() <= 1e-3 * np.abs(got[live]).max()


def test_tensor_core_conv_matches_cuda_core(gpu_lib):
    """tcgen05 implicit-GEMM convolution (128-voxel tiles) vs the CUDA-core
    kernel on the same bf16 inputs: forward outputs and parameter gradients."""
    n = 128
    net, p = _net(n)
    x = _inputs(n, 11)
    g3 = np.random.default_rng(9).normal(0, 1, (n, n, n, 3)).astype(np.float32)
    net.tensor_cores(True)
    out_tc = net.forward_host(x)
    gr_tc = net.backward_host(x, g3)
    net.tensor_cores(False)
    out_s = net.forward_host(x)
    gr_s = net.backward_host(x, g3)
    assert np.abs(out_tc - out_s).max() <= 2e-2 * np.abs(out_s).max()
    assert np.corrcoef(out_tc.ravel(), out_s.ravel())[0, 1] > 0.99999
    rel = np.linalg.norm(gr_tc - gr_s) / np.linalg.norm(gr_s)
    assert rel < 1e-2, rel
    # and against the oracle on a slab (forward only; the oracle is O(N^3))
    want = CR.forward(x, p, dtype=__import__("torch").float32)[0].numpy()
    assert np.abs(out_tc - want).max() <= 2e-2 * np.abs(want).max()


def test_training_on_pm_pairs_reduces_force_error(gpu_lib, bbks_table):
    """Pairs from the method itself: factor-1 (coarse) vs factor-3 (fine) PM
    forces on the same particles.  After training, the corrected coarse
    force is closer to the fine force on held-out particles than the plain
    coarse force is."""
    from cola_halo_b200 import Simulation
    from cola_halo_b200.learned import ConvNet, copy_particles
    from cola_halo_b200.schedule import Schedule
    from tests.helpers import lattice_particles
    nc, L, om = 32, 100.0, 0.273
    sched = Schedule.linear(0.1, 1.0, 6)
    fine = Simulation(nc, 3 * nc, L, om)
    coarse = Simulation(nc, nc, L, om)
    net = ConvNet(nc, seed=1)
    net.set_scales(1.0, 1.0, 1.0)

    def trajectory(seed):
        p = lattice_particles(nc, L, seed, om, sched.a_init, bbks_table)
        fine.set_particles(p, sched.a_init, sched.a_init)
        states = []
        for i in range(1, sched.nloop):
            _, _, avel1, apos1 = sched.times(i)
            fine.move()
            fine.forces()
            states.append(fine.get_particles())
            fine.kick(avel1)
            fine.drift(apos1)
        return states

    train = trajectory(1) + trajectory(2)
    test = trajectory(3)[-2:]
    losses = []
    for epoch in range(40):
        for s in train:
            fine.set_particles(s, 0.5, 0.5)
            copy_particles(coarse, fine)
            losses.append(net.train_step(coarse, fine, 3e-3))
    assert np.mean(losses[-len(train):]) < 0.5 * np.mean(losses[:len(train)])

    def errs(s):
        fine.set_particles(s, 0.5, 0.5)
        fine.forces()
        ff = fine.get_forces()
        copy_particles(coarse, fine)
        coarse.forces()
        fc = coarse.get_forces()
        net.forces(coarse)
        fl = coarse.get_forces()
        return (np.sqrt(np.mean((fc - ff) ** 2)), np.sqrt(np.mean((fl - ff) ** 2)))
    for s in test:
        e_plain, e_learned = errs(s)
        assert e_learned < 0.9 * e_plain, (e_plain, e_learned)


def test_line_ring_conv_bit_identical(gpu_lib):
    """At 128^3 the tensor-core convolutions reuse input lines along y (the
    line ring); its MMAs and operands are those of the one-stage kernel,
    so forward outputs are bit-identical.  The parameter gradients agree to
    the rounding of the weight gradient's float atomics, whose order varies
    from run to run."""
    from cola_halo_b200.learned import ConvNet
    n = 128
    rng = np.random.default_rng(5)
    x = rng.normal(0, 1, (n, n, n, 2)).astype(np.float32)
    g = rng.normal(0, 1, (n, n, n, 3)).astype(np.float32)
    net = ConvNet(n, seed=3)
    out, grads = [], []
    try:
        for v in (1, 2):
            assert gpu_lib.cg_net_set_conv_variant(v) == 0
            out.append(net.forward_host(x))
            grads.append(net.backward_host(x, g))
    finally:
        gpu_lib.cg_net_set_conv_variant(-1)
    np.testing.assert_array_equal(out[0], out[1])
    np.testing.assert_allclose(grads[0], grads[1], rtol=1e-4, atol=1e-6 * np.abs(grads[0]).max())
    assert gpu_lib.cg_net_set_conv_variant(5) != 0
    net.close()
