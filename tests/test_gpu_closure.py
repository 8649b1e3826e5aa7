"""Learned subgrid closure on the tensor cores (tcgen05, BF16 operands, F32
accumulation in tensor memory), through the C ABI, against host products."""
import ctypes

import numpy as np
import pytest

from compchan3dmpi_b200 import _lib

pytestmark = pytest.mark.gpu


def to_bf16_bits(x):
    """float -> BF16 bit patterns, round to nearest even."""
    b = np.ascontiguousarray(x, dtype=np.float32).view(np.uint32).astype(np.uint64)
    b = (b + 0x7FFF + ((b >> 16) & 1)) >> 16
    return b.astype(np.uint16)


def from_bf16_bits(b):
    return (np.asarray(b, dtype=np.uint32) << 16).view(np.float32).astype(np.float64)


@pytest.mark.parametrize("K,N", [(16, 16), (16, 64), (64, 16), (64, 64), (128, 128), (32, 256)])
def test_umma_gemm_matches_host_product(K, N):
    rng = np.random.default_rng(K * 1000 + N)
    A = to_bf16_bits(rng.standard_normal((128, K)))
    B = to_bf16_bits(rng.standard_normal((N, K)))
    D = np.zeros((128, N), dtype=np.float32)
    L = _lib.load()
    r = L.chan_selftest_umma(A.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                             B.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16)),
                             D.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), K, N, 0)
    assert r == 0
    ref = from_bf16_bits(A) @ from_bf16_bits(B).T
    err = np.max(np.abs(D - ref)) / np.max(np.abs(ref))
    assert err < 1e-6, err


# ----------------------------------------------------------------- the closure
from chan_cases import make_case                       # noqa: E402
from compchan3dmpi_b200 import Channel, ChanError, RK2  # noqa: E402
from compchan3dmpi_b200.closure import Closure, attach, closure_flag, run_with_fallback  # noqa: E402
from oracle import closure_oracle as C                  # noqa: E402


def _random_closure(seed=5, scale=0.4, ysd=1.0):
    rng = np.random.default_rng(seed)
    params = (rng.standard_normal(C.N_PARAM) * scale).astype(np.float32)
    norm = np.concatenate([rng.standard_normal(13) * 0.1, 0.5 + rng.random(13),
                           rng.standard_normal(9) * 0.1, ysd * (0.5 + rng.random(9))]).astype(np.float32)
    cl = Closure(capacity=0)
    cl.norm = norm
    cl.params = params
    return cl, params, norm


def test_mlp_inference_matches_oracle():
    cl, params, norm = _random_closure()
    X = np.random.default_rng(1).standard_normal((1000, 13)).astype(np.float32)
    Y = cl.infer(X)
    ref, _ = C.forward(params, norm, X)
    err = np.max(np.abs(Y - ref)) / np.max(np.abs(ref))
    assert err < 2e-2, err      # BF16 activations: roundings may differ at a boundary
    assert np.mean(np.abs(Y - ref)) / np.mean(np.abs(ref)) < 2e-3


def test_mlp_gradients_match_oracle():
    """One training step's loss and gradients (forward, the two data-gradient
    and three weight-gradient products on the tensor cores) against the
    oracle's float64 restatement with the same BF16 roundings; 300 rows, so
    the last tile is partly empty.

    Tolerance: device and oracle round the same quantities to BF16 at the same
    places.  They differ only where the order of an F32 accumulation (tensor
    core against numpy, relative differences ~1e-7) moves a value across a
    BF16 rounding boundary (half an ulp is 2^-9 ~ 2e-3 relative), which
    changes that element by one BF16 ulp.  Such flips touch a fraction of
    order 1e-4 of the elements, so a gradient's relative L2 error is ~1e-4
    (9.6e-5 measured over the whole gradient); the bound per parameter group
    is 2e-3, 20 times that."""
    cl, params, norm = _random_closure(seed=9)
    rng = np.random.default_rng(2)
    X = rng.standard_normal((300, 13)).astype(np.float32)
    T = rng.standard_normal((300, 9)).astype(np.float32)
    loss, g = cl.grad(X, T)
    lo, go = C.grad(params, norm, X, T)
    assert abs(loss - lo) <= 1e-3 * lo
    for name, a, b in (("W1", C.OFF_W1, C.OFF_B1), ("b1", C.OFF_B1, C.OFF_W2), ("W2", C.OFF_W2, C.OFF_B2),
                       ("b2", C.OFF_B2, C.OFF_W3), ("W3", C.OFF_W3, C.OFF_B3), ("b3", C.OFF_B3, C.N_PARAM)):
        e = np.linalg.norm(g[a:b] - go[a:b]) / np.linalg.norm(go[a:b])
        assert e < 2e-3, (name, e)


def test_adam_step_and_training_reduce_the_loss():
    """One Adam step equals the oracle's on the device's own gradient; then
    training on a smooth synthetic map lowers the loss several times over."""
    rng = np.random.default_rng(4)
    X = rng.standard_normal((16384, 13)).astype(np.float32)
    A = rng.standard_normal((13, 9)) * 0.5
    T = (np.tanh(X @ A) + 0.1 * X[:, :9] ** 2).astype(np.float32)
    cl = Closure(capacity=20000)
    cl.add_data(X, T)
    assert cl.count == 16384
    cl.fit_normalization()
    cl.init(seed=11)
    p0 = cl.params.astype(np.float64)
    _, g = cl.grad(X[:2048], T[:2048])
    # one epoch of one batch over the first 2048 rows equals one Adam step of that gradient
    cl2 = Closure(capacity=2048)
    cl2.add_data(X[:2048], T[:2048])
    cl2.norm = cl.norm
    cl2.params = p0
    cl2.train(1, batch=2048, lr=1e-3, seed=1)
    w1, _, _ = C.adam(p0, np.zeros_like(p0), np.zeros_like(p0), g.astype(np.float64), 1, 1e-3)
    assert np.max(np.abs(cl2.params - w1)) <= 1e-6 + 1e-5 * np.max(np.abs(w1))
    losses = cl.train(30, batch=1024, lr=2e-3, seed=3)
    assert np.all(np.isfinite(losses))
    assert losses[-1] < losses[0] / 3, losses


def _dns_case():
    p, x3, jac, inv, var = make_case(nP=(24, 18, 19), mesh="tanh", beta=2.2, rk=RK2, istat=2, quantize=False)
    return p, x3, jac, inv, var


def test_sampling_matches_oracle():
    p, x3, jac, inv, var = _dns_case()
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    g.step(4)
    cl = Closure(capacity=10000)
    n = cl.sample(g, strides=(2, 2, 2), width=2)
    X, T = cl.data()
    assert X.shape[0] == n > 0
    tau, s1, _, _ = g.stats()
    Xo, To = C.sample(g.download(), x3, p.dx, p.dy, p.Re, 2, 2, 2, 2, tau, s1)
    assert Xo.shape == X.shape
    for a, b in ((X, Xo), (T, To)):
        for c in range(a.shape[1]):
            scale = max(np.max(np.abs(b[:, c])), 1e-30)
            assert np.max(np.abs(a[:, c] - b[:, c])) <= 1e-5 * scale, c


def test_closure_source_matches_oracle():
    """A stage with the closure minus the same stage without it is cdt times
    the oracle's closure source at every interior point."""
    p, x3, jac, inv, var = _dns_case()
    cl, params, norm = _random_closure(seed=21, scale=0.3, ysd=0.01)
    a = Channel(p, x3, jac, inv)
    b = Channel(p, x3, jac, inv)
    attach(a, cl, True)
    for ch in (a, b):
        ch.init_sol_v(var)
        ch.stage(1)
    va, vb = a.download(), b.download()
    dq = np.stack([va[0] * va[m] - vb[0] * vb[m] for m in (1, 2, 3, 4)])[:, 1:-1, 1:-1, 1:-1]
    n1, n2, n3 = p.nP
    czh = np.zeros(n3 + 2)
    czh[1:n3 + 1] = 0.5 / p.dXi * np.asarray(inv)
    S = C.source(var, x3, czh, p.dx, p.dy, p.Re, p.gama, params, norm, (0.0, 0.0), np.zeros((7, n3)))
    cdt = 0.5 * p.dt
    for r in range(4):
        scale = np.max(np.abs(S[r]))
        assert scale > 0
        assert np.max(np.abs(dq[r] - cdt * S[r])) <= 2e-2 * cdt * scale, r
    assert np.array_equal(va[0], vb[0])   # no mass source
    assert closure_flag(a) == 0


def test_closure_refused_on_mixed_contexts():
    p, x3, jac, inv, var = _dns_case()
    cl, _, _ = _random_closure()
    m = Channel(p.with_(mixed=True, rk_scheme=3), x3, jac, inv)
    with pytest.raises(ChanError):
        attach(m, cl, True)


def test_divergent_closure_falls_back_to_the_plain_method(tmp_path):
    """Weights scaled up 1e3 drive the outputs past their limit: the run
    restores the last good checkpoint and finishes with the plain method."""
    p, x3, jac, inv, var = _dns_case()
    cl, params, norm = _random_closure(seed=33)
    cl.params = params * 1e3
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    rep = run_with_fallback(g, cl, steps=12, check_every=4, workdir=str(tmp_path))
    assert rep["fallback_step"] is not None and rep["reason"] is not None
    assert rep["plain_failed"] is None
    assert g.nstep == 12 and g.status() == 0
    assert np.all(np.isfinite(g.download()))
    # the plain method from the same start gives the same state
    h = Channel(p, x3, jac, inv)
    h.init_sol_v(var)
    h.step(12)
    assert np.array_equal(g.download(), h.download())


def test_closure_once_per_step_and_every_stage():
    """Stage 1 is the same in both modes; over whole steps the two differ only
    by holding the first stage's source (both stay finite and close)."""
    p, x3, jac, inv, var = _dns_case()
    cl, params, norm = _random_closure(seed=21, scale=0.3, ysd=0.01)
    a = Channel(p, x3, jac, inv)
    b = Channel(p, x3, jac, inv)
    attach(a, cl, True)
    attach(b, cl, True, every_stage=True)
    for ch in (a, b):
        ch.init_sol_v(var)
        ch.stage(1)
    assert np.array_equal(a.download(), b.download())
    for ch in (a, b):
        ch.init_sol_v(var)
        ch.step(5)
    va, vb = a.download(), b.download()
    assert np.all(np.isfinite(va)) and np.all(np.isfinite(vb))
    assert not np.array_equal(va, vb)
    assert np.max(np.abs(va - vb)) < 5e-2 * np.max(np.abs(vb))


def test_fallback_without_a_workdir_leaves_no_files(monkeypatch, tmp_path):
    """With no workdir the last good checkpoint lives in a temporary directory
    that is removed on return."""
    import tempfile
    monkeypatch.setattr(tempfile, "tempdir", str(tmp_path))
    p, x3, jac, inv, var = _dns_case()
    cl, params, norm = _random_closure(seed=33)
    cl.params = params * 1e3
    g = Channel(p, x3, jac, inv)
    g.init_sol_v(var)
    rep = run_with_fallback(g, cl, steps=8, check_every=4)
    assert rep["reason"] is not None and g.nstep == 8
    assert list(tmp_path.iterdir()) == []

