"""torch extension on the GPU: adjointness, the analytic Poisson gradient,
and the unrolled relaxed MLEM against FP64 central finite differences of the
oracle (small workload, K = 10, 64 random directions, step 1e-3 relative,
tolerance 1e-3 relative L2 over the directions)."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

from mlem_b200 import api, synth, torch_ext  # noqa: E402

import oracle_bind as ob  # noqa: E402

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small(golden):
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    ctx = api.Context.from_matrix(m)
    yield m, sino, ctx
    ctx.close()


def test_projector_adjoint(small):
    m, sino, ctx = small
    g = torch.Generator(device="cpu").manual_seed(0)
    x = torch.rand(m.n_cols, generator=g).cuda()
    y = torch.rand(m.n_rows, generator=g).cuda()
    lhs = torch.dot(torch_ext.forward_project(x, ctx).double(), y.double())
    rhs = torch.dot(x.double(), torch_ext.back_project(y, ctx).double())
    assert abs(float(lhs - rhs)) <= 1e-5 * abs(float(lhs))
    # batched frames give the same per-frame results
    X = torch.rand(3, m.n_cols, generator=g).cuda()
    Y = torch_ext.forward_project(X, ctx)
    for b in range(3):
        assert torch.allclose(Y[b], torch_ext.forward_project(X[b].contiguous(), ctx), rtol=1e-6, atol=0)


def test_poisson_gradient_matches_analytic(small):
    m, sino, ctx = small
    x0 = synth.phantom(32, 32, 16, 5, 77).astype(np.float32) + 0.5
    x = torch.tensor(x0, device="cuda", requires_grad=True)
    s = torch.tensor(sino, device="cuda", dtype=torch.float32)
    f = torch_ext.forward_project(x, ctx)
    safe = torch.where(f > 0, f, torch.ones_like(f))
    loss = torch.sum(torch.where(f > 0, f - s * torch.log(safe), f))
    loss.backward()
    want = ob.poisson_grad_f64(m, sino, x0.astype(np.float64))
    assert ob.rel_l2(x.grad.cpu().numpy(), want) <= 1e-5


def _loss64(m, sino, x0, omega, x_true):
    xk = ob.mlem_relaxed_f64(m, sino, x0, omega)
    return float(np.mean((xk - x_true) ** 2))


@pytest.mark.parametrize("keep_bytes", [2 << 30, 0])
def test_unrolled_mlem_gradients_match_fp64_finite_differences(small, keep_bytes):
    """Both ways of the backward pass: the row sums and update factors kept
    by the forward pass, and (keep_bytes 0) recomputed from the images."""
    m, sino, ctx = small
    K = 10
    x_true = synth.phantom(32, 32, 16, 5, 0).astype(np.float64)
    norm = ob.column_sums(m)
    x0 = np.full(m.n_cols, ob.init_value(norm, sino), np.float64)
    omega = 1.0 + 0.05 * np.sin(np.arange(K))

    xt = torch.tensor(x0, device="cuda", dtype=torch.float32, requires_grad=True)
    wt = torch.tensor(omega, device="cuda", dtype=torch.float32, requires_grad=True)
    st = torch.tensor(sino, device="cuda")
    xK = torch_ext.unrolled_mlem(xt, wt, st, ctx, keep_bytes=keep_bytes)
    loss = torch.mean((xK.double() - torch.tensor(x_true, device="cuda")) ** 2)
    loss.backward()
    gx = xt.grad.double().cpu().numpy()
    gw = wt.grad.double().cpu().numpy()
    # forward agrees with the FP64 oracle
    assert ob.rel_l2(xK.detach().cpu().numpy(), ob.mlem_relaxed_f64(m, sino, x0, omega)) <= 1e-4

    rng = np.random.default_rng(1)
    eps = 1e-3
    d_gpu, d_fd = [], []
    for _ in range(64):
        v = rng.standard_normal(m.n_cols)
        v *= np.linalg.norm(x0) / np.linalg.norm(v)
        lp = _loss64(m, sino, x0 + eps * v, omega, x_true)
        lm = _loss64(m, sino, x0 - eps * v, omega, x_true)
        d_fd.append((lp - lm) / (2 * eps))
        d_gpu.append(float(gx @ v))
    d_gpu, d_fd = np.array(d_gpu), np.array(d_fd)
    assert np.linalg.norm(d_gpu - d_fd) <= 1e-3 * np.linalg.norm(d_fd)

    w_gpu, w_fd = [], []
    for _ in range(16):
        v = rng.standard_normal(K)
        v *= np.linalg.norm(omega) / np.linalg.norm(v)
        lp = _loss64(m, sino, x0, omega + eps * v, x_true)
        lm = _loss64(m, sino, x0, omega - eps * v, x_true)
        w_fd.append((lp - lm) / (2 * eps))
        w_gpu.append(float(gw @ v))
    w_gpu, w_fd = np.array(w_gpu), np.array(w_fd)
    assert np.linalg.norm(w_gpu - w_fd) <= 1e-3 * np.linalg.norm(w_fd)


@pytest.mark.parametrize("keep_bytes", [2 << 30, 0])
def test_unrolled_mlem_gradients_finite_with_tiny_projections(small, keep_bytes):
    """Rows with zero counts whose projection is tiny but nonzero (a start
    image of 1e-25: f^2 underflows to 0 in float32) give no gradient through
    calcCorrel instead of 0 / 0."""
    m, sino, ctx = small
    rng = np.random.default_rng(4)
    s = sino.copy()
    s[rng.random(s.size) < 0.3] = 0
    K = 3
    xt = torch.full((m.n_cols,), 1e-25, device="cuda", dtype=torch.float32, requires_grad=True)
    wt = torch.ones(K, device="cuda", dtype=torch.float32, requires_grad=True)
    x_true = torch.tensor(synth.phantom(32, 32, 16, 5, 0), device="cuda", dtype=torch.float32)
    xK = torch_ext.unrolled_mlem(xt, wt, torch.tensor(s, device="cuda"), ctx, keep_bytes=keep_bytes)
    loss = torch.mean((xK - x_true) ** 2)
    loss.backward()
    assert torch.isfinite(xK).all()
    assert torch.isfinite(xt.grad).all() and torch.isfinite(wt.grad).all()
    assert float(wt.grad.abs().sum()) > 0


@pytest.mark.parametrize("flags", [0, api.FLAG_NATURAL_LAYOUT | api.FLAG_NO_ROW_ORDER])
def test_backward_pass_kernels_against_the_oracle(golden, flags):
    """mlem_ratio_rows_d and mlem_adjoint_update_d (the backward pass's two
    one-pass kernels) against the oracle's projections, in the Morton layout
    with sorted rows and in natural order with file-order rows."""
    m, sino, iters, gold, _ = golden.case("plain_small_it10")
    rng = np.random.default_rng(8)
    s = np.ascontiguousarray(sino, np.int32).copy()
    s[rng.random(m.n_rows) < 0.3] = 0
    x = rng.uniform(0.5, 2.0, m.n_cols).astype(np.float32)
    du = rng.normal(0.0, 1.0, m.n_cols).astype(np.float32)
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    with api.Context.from_matrix(m, flags=flags) as ctx:
        xs, dus, sd = (torch.from_numpy(a).to(dev) for a in (x, du, s))
        rows = torch.empty(m.n_rows, dtype=torch.float32, device=dev)
        u = torch.empty(m.n_cols, dtype=torch.float32, device=dev)
        ctx.ratio_rows_d(xs.data_ptr(), sd.data_ptr(), rows.data_ptr(), u.data_ptr(), st)
        a = torch.empty_like(u)
        ctx.adjoint_update_d(dus.data_ptr(), sd.data_ptr(), rows.data_ptr(), a.data_ptr(), st)
        torch.cuda.synchronize()
        f_got, u_got, a_got = rows.cpu().numpy(), u.cpu().numpy(), a.cpu().numpy()
    f = ob.fwproj(m, x)
    live = s != 0
    assert ob.rel_l2(f_got[live], f[live]) <= 1e-5
    assert not f_got[~live].any()
    assert ob.rel_l2(u_got, ob.bkproj(m, ob.correl(f, s))) <= 1e-5
    f64 = f.astype(np.float64)
    dc = ob.fwproj(m, du).astype(np.float64)
    ok = live & (f64 != 0)
    df = np.where(ok, -(dc * (s / np.where(ok, f64, 1.0))) / np.where(ok, f64, 1.0), 0.0)
    assert ob.rel_l2(a_got, ob.bkproj(m, df.astype(np.float32))) <= 1e-5


def test_backward_pass_kernels_on_an_odd_matrix():
    """Empty rows, a row far longer than one load batch, duplicate columns,
    zero values and odd sizes through both backward-pass kernels."""
    from mlem_b200 import formats
    rng = np.random.default_rng(17)
    R, C = 777, 333
    lens = rng.integers(0, 40, R)
    lens[::9] = 0
    lens[5] = 10000
    row_end = np.cumsum(lens).astype(np.uint64)
    el = np.zeros(int(row_end[-1]), formats.ELEM_DTYPE)
    el["index"] = rng.integers(0, C, el.size)
    el["value"] = rng.uniform(0.0, 1.7, el.size).astype(np.float32)
    el["value"][::13] = 0.0
    m = formats.Csr4(R, C, row_end, el)
    s = rng.poisson(3.0, R).astype(np.int32)
    x = rng.uniform(0.5, 2.0, C).astype(np.float32)
    du = rng.normal(0.0, 1.0, C).astype(np.float32)
    dev = torch.device("cuda", 0)
    st = torch.cuda.current_stream().cuda_stream
    with api.Context.from_matrix(m) as ctx:
        xs, dus, sd = (torch.from_numpy(a).to(dev) for a in (x, du, s))
        rows = torch.empty(R, dtype=torch.float32, device=dev)
        u = torch.empty(C, dtype=torch.float32, device=dev)
        a = torch.empty(C, dtype=torch.float32, device=dev)
        ctx.ratio_rows_d(xs.data_ptr(), sd.data_ptr(), rows.data_ptr(), u.data_ptr(), st)
        ctx.adjoint_update_d(dus.data_ptr(), sd.data_ptr(), rows.data_ptr(), a.data_ptr(), st)
        torch.cuda.synchronize()
        f_got, u_got, a_got = rows.cpu().numpy(), u.cpu().numpy(), a.cpu().numpy()
    f = ob.fwproj(m, x)
    live = s != 0
    assert ob.rel_l2(f_got[live], f[live]) <= 1e-5
    assert ob.rel_l2(u_got, ob.bkproj(m, ob.correl(f, s))) <= 1e-5
    f64 = f.astype(np.float64)
    dc = ob.fwproj(m, du).astype(np.float64)
    ok = live & (f64 != 0)
    df = np.where(ok, -(dc * (s / np.where(ok, f64, 1.0))) / np.where(ok, f64, 1.0), 0.0)
    assert ob.rel_l2(a_got, ob.bkproj(m, df.astype(np.float32))) <= 1e-5
