"""The learned substep: tensor-core (tcgen05) inference against the FP32 forward of the same
weights, training on implicit-solver pairs, and the surrogate-with-fallback substep (FP64
conservation, fallback cells equal to the implicit solve, judged error)."""
import os

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from tiger_nga_b200 import capi, states  # noqa: E402
from tiger_nga_b200.mechanism import load  # noqa: E402

pytestmark = pytest.mark.gpu
P = 101325.0


def pairs(chem, n, seed):
    m = load(chem.mechanism)
    sol, _ = states.chem_state(m, n, seed, "CH4", grid=(n, 1, 1), progress="beta22", T_range=(300.0, 2400.0))
    rng = np.random.default_rng(seed)
    dts = 10 ** rng.uniform(-7, -5, n)
    s0 = torch.from_numpy(sol).cuda()
    s1 = s0.clone()
    d = torch.from_numpy(dts).cuda()
    chem.substep(s1, d, P)
    return s0, s1, d


@pytest.fixture(scope="module")
def trained():
    chem = capi.FiniteChem("grimech30", "fp64")
    s0, s1, d = pairs(chem, 32768, 11)
    sur = capi.Surrogate(chem, judge_cells=256)
    losses = sur.train(s0, s1, d, P, epochs=12, batch=2048, lr=2e-3)
    return chem, sur, losses


def test_training_reduces_loss(trained):
    _, _, losses = trained
    assert np.isfinite(losses).all() and losses[-1] < 0.5 * losses[0]


def test_tensor_core_chain_matches_fp32_forward(trained):
    chem, sur, _ = trained
    s0, _, d = pairs(chem, 4099, 12)  # ragged: 32 full tiles + 3 rows
    Y_tc = sur.infer(s0, d, P)
    X = sur.features(s0, d, P)
    Y32 = sur.forward_f32(X)
    torch.cuda.synchronize()
    a, b = Y_tc.cpu().numpy()[:, :sur.n_out], Y32.cpu().numpy()[:, :sur.n_out]
    # BF16 operands, FP32 accumulation: agreement at the BF16 rounding level of the layer
    # activations, which are O(1) (outputs whose own range is smaller -- trace species under the
    # shared output scale -- are compared against 1)
    scale = np.maximum(np.abs(b).max(axis=0), 1.0)
    assert np.isfinite(a).all()
    assert np.max(np.abs(a - b) / scale) < 0.05
    assert np.median(np.abs(a - b) / scale) < 0.005


def _bf16(t):
    return t.to(torch.bfloat16).to(torch.float32)


def _bf16_chain(sur, X):
    """FP32 forward of member 0 with the tensor-core chain's roundings: the features, the
    weights and every hidden activation rounded to BF16, products accumulated in FP32, bias and
    GELU (tanh form) in FP32."""
    flat = torch.from_numpy(sur.params()).cuda()
    off, fi, h = 0, sur.in_pad, _bf16(X)
    for layer in range(sur.cfg.layers + 1):
        fo = sur.out_pad if layer == sur.cfg.layers else sur.cfg.hidden
        W = flat[off:off + fo * fi].view(fo, fi)
        b = flat[off + fo * fi:off + fo * fi + fo]
        off += fo * fi + fo
        z = torch.matmul(h, _bf16(W).T) + b
        h = z if layer == sur.cfg.layers else _bf16(torch.nn.functional.gelu(z, approximate="tanh"))
        fi = fo
    return h


def test_tensor_core_chain_matches_bf16_rounded_forward(trained):
    """The tcgen05 chain against a forward that rounds exactly where the kernel rounds: what is
    left is FP32 summation order, the kernel's GELU and the BF16 rounding flips they cause (a few
    BF16 ulps, 2^-8 each, at the largest outputs). A wrong operand layout, descriptor or bias
    would show as O(1) errors."""
    chem, sur, _ = trained
    s0, _, d = pairs(chem, 4099, 16)
    Y_tc = sur.infer(s0, d, P)
    ref = _bf16_chain(sur, sur.features(s0, d, P))
    torch.cuda.synchronize()
    a, b = Y_tc[:, :sur.n_out].double(), ref[:, :sur.n_out].double()
    scale = torch.clamp(b.abs().amax(0), min=1.0)
    err = ((a - b).abs() / scale).cpu().numpy()
    assert np.isfinite(err).all()
    assert err.max() < 1e-2, err.max()
    assert np.median(err) < 5e-4, np.median(err)


def test_inference_wait_limit_runs_out_and_the_next_call_succeeds(trained):
    """The inference kernel's bounded waits: with a short poll limit and one withheld completion
    signal per CTA the wait gives up, the kernel drains its copies and MMAs, frees its tensor
    memory and reports the timeout (TNG_ERR_CUDA); the next normal call on the same surrogate
    returns the same predictions as before."""
    chem, sur, _ = trained
    s0, _, d = pairs(chem, 4099, 17)
    good = sur.infer(s0, d, P).clone()
    sur.debug_waits(wait_limit=2000, fault=1)
    try:
        with pytest.raises(capi.ChemError, match="timed out"):
            sur.infer(s0, d, P)
    finally:
        sur.debug_waits(0, 0)
    again = sur.infer(s0, d, P)
    torch.cuda.synchronize()
    assert torch.equal(again, good)


def test_surrogate_substep_conserves_and_falls_back(trained):
    chem, sur, _ = trained
    m = load("grimech30")
    s0, s_ref, d = pairs(chem, 8192, 13)
    x = s0.clone()
    st = sur.substep(x, d, P)
    assert st["cells"] == 8192 and st["accepted"] + st["fallback"]["cells"] == 8192
    assert st["judged"] == 256 and np.isfinite(st["judge_max_rel_dT"])
    out, ref, ini = x.cpu().numpy(), s_ref.cpu().numpy(), s0.cpu().numpy()
    assert np.isfinite(out).all()
    # cells that fell back equal the implicit solve exactly
    same = np.all(out == ref, axis=0)
    assert same.sum() >= st["fallback"]["cells"]
    # accepted cells: mass and elements conserved by the FP64 projection (the implicit solve
    # itself drifts at ~1e-9 because the reference's molar masses are single-precision literals)
    acc = ~same
    assert acc.sum() > 0
    rho0, rho1 = ini[:-1].sum(0), out[:-1].sum(0)
    assert np.max(np.abs(rho1 - rho0)[acc] / rho0[acc]) < 1e-12  # mass
    E = m.elem / m.wmol[None, :]
    el0, el1 = E @ (ini[:-1] / rho0), E @ (out[:-1] / rho1)
    # element conservation: exact up to the final renormalisation sum(Y) = 1, which moves E.Y by
    # sum(dY) ~ 1e-8 because the single-precision molar masses are not exact sums of atomic masses
    scale = np.maximum(el0.max(axis=1, keepdims=True), 1e-6)  # elements absent from the batch: absolute
    assert np.max((np.abs(el1 - el0) / scale)[:, acc]) < 1e-7


def test_save_load_roundtrip(trained, tmp_path):
    chem, sur, _ = trained
    path = str(tmp_path / "gri.tngs")
    sur.save(path)
    sur2 = capi.Surrogate(chem, judge_cells=0)
    sur2.load(path)
    s0, _, d = pairs(chem, 1024, 14)
    assert torch.equal(sur.infer(s0, d, P), sur2.infer(s0, d, P))
    assert np.array_equal(sur.params(), sur2.params())
