"""Every Backend method on the GPU against the CPU oracle, on scaled Netlib problems and
deterministic pseudo-random vectors: the protocol of crates/saddlepoint-cuda/tests/ops.rs:53-146
(vectors in [-2, 2] with every fifth zero, tau = 0.37, sigma = 1.9, w = 0.8, rho = 1;
max|a-b|/(1+max|a|) < 1e-12 for vectors, |a-b|/(1+max(|a|,|b|)) < 1e-11 for scalars).

On top of the reference's tolerances, the element-wise steps must match bit for bit (the
library is built without FMA contraction) and so must SpMV rows short enough to be summed
by one thread in column order."""
import numpy as np
import pytest

import oracle
from conftest import netlib_lp, xorshift_vector

pytestmark = pytest.mark.gpu

NAMES = ["afiro", "israel", "25fv47", "80bau3b", "perold"]


def close(what, a, b):
    err = abs(a - b) / (1.0 + max(abs(a), abs(b)))
    assert err < 1e-11, f"{what}: cpu {a} vs gpu {b} (relative {err:.2e})"


def close_vec(what, a, b):
    assert len(a) == len(b), what
    scale = 1.0 + (np.max(np.abs(a)) if len(a) else 0.0)
    err = (np.max(np.abs(a - b)) if len(a) else 0.0) / scale
    assert err < 1e-12, f"{what}: max relative difference {err:.2e}"


def short_rows(rp, limit=32):
    lens = np.diff(rp)
    return lens <= limit


@pytest.mark.parametrize("name", NAMES)
def test_backend_ops_match_cpu(name, gpu_backend):
    import saddlepoint_b200 as sp

    gpu = gpu_backend
    cpu = oracle.CpuBackend()
    lp = netlib_lp(name)
    s = oracle.scaled_problem(lp)
    m, n = s.nrows, s.ncols
    pc = cpu.load(s)
    scaled = sp.ScaledProblem(m, n, s.a, s.at, s.c, s.lc, s.uc, s.lv, s.uv, s.row_scale, s.col_scale,
                              s.bound_scale, s.obj_scale)
    pg = gpu.load(scaled)
    up, down = gpu.upload, gpu.download

    x, y = xorshift_vector(n, 1), xorshift_vector(m, 2)
    xa, ya = xorshift_vector(n, 3), xorshift_vector(m, 4)
    gx, gy, gxa, gya = up(x), up(y), up(xa), up(ya)

    # SpMV
    cm = cpu.spmv(pc, x)
    gm = up(np.zeros(m))
    gpu.spmv(pg, gx, gm)
    close_vec(f"{name} spmv", cm, down(gm))
    short = short_rows(s.a[0])
    assert np.array_equal(cm[short], down(gm)[short]), "short rows must be bit-exact"
    cn = cpu.spmv_t(pc, y)
    gn = up(np.zeros(n))
    gpu.spmv_t(pg, gy, gn)
    close_vec(f"{name} spmv_t", cn, down(gn))
    assert np.array_equal(cn[short_rows(s.at[0])], down(gn)[short_rows(s.at[0])])

    # steps
    tau = 0.37
    ct, cb = cpu.primal_step(pc, x, cn, tau)
    gt, gb = up(np.zeros(n)), up(np.zeros(n))
    gpu.primal_step(pg, gx, up(cn), tau, gt, gb)
    assert np.array_equal(ct, down(gt)) and np.array_equal(cb, down(gb)), f"{name} primal_step"
    sigma = 1.9
    cyt = cpu.dual_step(pc, y, cm, sigma)
    gyt = up(np.zeros(m))
    gpu.dual_step(pg, gy, up(cm), sigma, gyt)
    assert np.array_equal(cyt, down(gyt)), f"{name} dual_step"
    cz = cpu.halpern_step(x, ct, xa, 0.8, 1.0)
    gz = up(x)
    gpu.halpern_step(gz, up(ct), gxa, 0.8, 1.0)
    assert np.array_equal(cz, down(gz)), f"{name} halpern_step"

    # vector helpers
    close(f"{name} distance_sq", cpu.distance_sq(x, xa), gpu.distance_sq(gx, gxa))
    close(f"{name} norm_sq", cpu.norm_sq(y), gpu.norm_sq(gy))
    close(f"{name} dot", cpu.dot(y, ya), gpu.dot(gy, gya))
    cs = cpu.sub(x, xa)
    gs = up(np.zeros(n))
    gpu.sub(gx, gxa, gs)
    assert np.array_equal(cs, down(gs))
    cs2 = cpu.scale(cs, -1.5)
    gpu.scale(gs, -1.5)
    assert np.array_equal(cs2, down(gs))

    # stats (projected iterate so bounds are active)
    gct = up(ct)
    gcm = up(cm)
    ps_c, ps_g = cpu.primal_stats(pc, ct, cm), gpu.primal_stats(pg, gct, gcm)
    close(f"{name} primal residual", ps_c[0], ps_g.residual_sq)
    close(f"{name} primal objective", ps_c[1], ps_g.objective)
    gcn = up(cn)
    ds_c, ds_g = cpu.dual_stats(pc, y, cn), gpu.dual_stats(pg, gy, gcn)
    close(f"{name} dual residual", ds_c[0], ds_g.residual_sq)
    close(f"{name} dual objective", ds_c[1], ds_g.objective)
    pr_c, pr_g = cpu.primal_ray_stats(pc, x, cm), gpu.primal_ray_stats(pg, gx, gcm)
    close(f"{name} primal ray objective", pr_c[0], pr_g.objective)
    close(f"{name} primal ray violation", pr_c[1], pr_g.violation_sq)
    close(f"{name} primal ray norm", pr_c[2], pr_g.norm_sq)
    dr_c, dr_g = cpu.dual_ray_stats(pc, y, cn), gpu.dual_ray_stats(pg, gy, gcn)
    close(f"{name} dual ray objective", dr_c[0], dr_g.objective)
    close(f"{name} dual ray violation", dr_c[1], dr_g.violation_sq)
    close(f"{name} dual ray norm", dr_c[2], dr_g.norm_sq)
    sd_c = cpu.step_dual_residual_sq(pc, x, ct, cn, cs2, tau)
    sd_g = gpu.step_dual_residual_sq(pg, gx, gct, gcn, gs, tau)
    close(f"{name} step dual residual", sd_c, sd_g)

    # copy and round trip
    gc = up(np.zeros(n))
    gpu.copy(gx, gc)
    assert np.array_equal(down(gc), x)


def test_reductions_are_deterministic(gpu_backend):
    gpu = gpu_backend
    v = xorshift_vector(300_000, 7)
    g = gpu.upload(v)
    r = [gpu.norm_sq(g) for _ in range(3)]
    assert r[0] == r[1] == r[2]
    assert abs(r[0] - float(np.dot(v, v))) <= 1e-12 * r[0]


def test_length_mismatch_is_an_error(gpu_backend):
    import saddlepoint_b200 as sp

    gpu = gpu_backend
    a, b = gpu.upload(np.ones(5)), gpu.upload(np.ones(6))
    with pytest.raises(sp.BackendError) as e:
        gpu.dot(a, b)
    assert e.value.code == 2
