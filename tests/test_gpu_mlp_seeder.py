"""The learned seeder (karam_seeder, KARAM_SEED_MLP) on the GPU.

- Its GEMM against an FP64 numpy product of the same BF16-rounded operands,
  within the FP32-accumulation bound K * 2^-23 * sum|a||b| (plus a small
  absolute floor), for every transpose combination and ragged sizes.
- Trained on plain-NR DC solutions of one set of config-2 MC instances, it
  seeds a held-out set: every seeded instance converges without the GMIN
  fallback, in fewer iterations than plain NR, and its solution meets the
  oracle tolerances (node voltages |dv| <= 1e-9 |v| + 1e-12 V, Norton branch
  currents within 1e-12 A).
"""
import numpy as np
import pytest

from karam_b200 import _abi as A
from karam_b200 import circuits

from test_gpu_parity import POLISH, branch_currents, scaled_err

pytestmark = pytest.mark.gpu


def bf16(x):
    u = np.ascontiguousarray(x, np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


@pytest.mark.parametrize("shape", [(67, 45, 130), (300, 260, 1030), (4, 512, 8)])
@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("tb", [False, True])
def test_bf16_gemm_matches_reference(product, ctx, ta, tb, shape):
    """The tcgen05 GEMM (TMA-staged BF16 operands, FP32 accumulation in tensor
    memory): several output tiles, K blocks beyond the ring of stages, ragged
    edges in M, N and K, every operand orientation."""
    rng = np.random.default_rng(11)
    M, N, K = shape
    a = rng.standard_normal((K, M) if ta else (M, K)).astype(np.float32)
    b = rng.standard_normal((N, K) if tb else (K, N)).astype(np.float32)
    c = product.bf16_gemm(a, b, trans_a=ta, trans_b=tb)
    oa = bf16(a).astype(np.float64)
    ob = bf16(b).astype(np.float64)
    oa = oa.T if ta else oa
    ob = ob.T if tb else ob
    ref = oa @ ob
    bound = K * 2.0**-23 * (np.abs(oa) @ np.abs(ob)) + 1e-6
    assert np.all(np.abs(c - ref) <= bound)


def _dc_batch(product, ctx, nl, inst, opts):
    prob = product.Problem(ctx, nl, max_instances=inst.n)
    prob.set_instances(inst)
    v, st = prob.solve_dc(opts)
    return prob, v, st


def test_mlp_seeder_trains_and_seeds_held_out_instances(product, ctx, port):
    nl = circuits.config2()
    train = circuits.mc_instances(nl, 512, first_instance=100000)
    held = circuits.mc_instances(nl, 64)
    plain = product.options(precision=A.PREC_MIXED, **POLISH)
    ptrain, _, st_train = _dc_batch(product, ctx, nl, train, plain)
    seeder = product.Seeder(ptrain, width=128, hidden_layers=2, init_seed=3)
    added = seeder.add_dc(ptrain)
    assert added == sum(s["status"] == A.ST_CONVERGED for s in st_train) and added >= 500
    first = seeder.train(epochs=1, batch=64, lr=2e-3, shuffle_seed=1)
    last = seeder.train(epochs=60, batch=64, lr=2e-3, shuffle_seed=2)
    assert np.isfinite(last) and last < first

    prob, v_plain, st_plain = _dc_batch(product, ctx, nl, held, plain)
    guess = seeder.predict(prob)
    assert np.max(np.abs(guess - v_plain)) < 0.05
    prob.set_seeder(seeder)
    v, st = prob.solve_dc(product.options(precision=A.PREC_MIXED, seeded=A.SEED_MLP, **POLISH))
    for i in range(held.n):
        assert st[i]["status"] == A.ST_CONVERGED and st[i]["seeded_ok"] == 1, (i, st[i])
        assert st[i]["iterations"] < st_plain[i]["iterations"]
    assert scaled_err(v, v_plain) <= 1.0
    for i in (0, held.n - 1):
        v_ref, st_ref = port.solve_dc(nl, held, i, linear_solver=1, **POLISH)
        assert scaled_err(v[i], v_ref) <= 1.0
        dI = np.abs(branch_currents(nl, v[i]) - branch_currents(nl, v_ref))
        assert dI.max() <= 1e-12, (i, dI)

    # a whole MC job (DC + transient) seeded by the network equals the plain one
    v0, st0 = prob.run_mc(held, 1e-12, 20, A.TRAN_BE, plain)
    r0 = prob.timing()["rounds"]
    v1, st1 = prob.run_mc(held, 1e-12, 20, A.TRAN_BE,
                          product.options(precision=A.PREC_MIXED, seeded=A.SEED_MLP, **POLISH))
    assert all(s["status"] == A.ST_CONVERGED for s in st0 + st1)
    assert scaled_err(v1, v0) <= 1.0
    assert prob.timing()["rounds"] < r0
    prob.set_seeder(None)
    seeder.close()


def test_mlp_seed_needs_a_trained_seeder(product, ctx):
    nl = circuits.config1()
    inst = circuits.mc_instances(nl, 4)
    prob = product.Problem(ctx, nl, max_instances=4)
    prob.set_instances(inst)
    opts = product.options(precision=A.PREC_FP64, seeded=A.SEED_MLP)
    with pytest.raises(product.KaramError) as e:
        prob.solve_dc(opts)
    assert e.value.code == A.KARAM_E_STATE
    seeder = product.Seeder(prob, width=16, hidden_layers=1)
    prob.set_seeder(seeder)
    with pytest.raises(product.KaramError):
        prob.solve_dc(opts)
    prob.set_seeder(None)
    other = product.Problem(ctx, circuits.config2(), max_instances=1)
    with pytest.raises(product.KaramError):
        other.set_seeder(seeder)


def _vdd_family(nl, first, n):
    """Config 5's instances: the chain's MC device variation and VDD ~ U(1.2, 2.0)."""
    inst = circuits.mc_instances(nl, n, first_instance=first)
    vdd = np.random.default_rng(first).uniform(1.2, 2.0, n)
    inst.vs_dc = np.stack([vdd, np.full(n, 0.9)], axis=1)
    return inst


def test_mlp_seeder_on_the_vdd_family_matches_oracle(product, ctx, port):
    """Config 5's family (the 256-stage chain, VIN 0.9 V, VDD ~ U(1.2, 2.0) and
    the MC variation): a seeder trained on plain-NR solutions of 2048
    instances seeds 32 held-out ones: the seeded solves converge on at least
    as many instances as plain NR, in fewer iterations on average, and where
    the oracle (FP64, sparse LU) converges too they reach its solution within
    the tolerance. (Outcomes of plain NR on this family depend on the
    precision: the bench compares them with the oracle's separately.)"""
    nl = circuits.inverter_chain(stages=256, vdd=1.8, vin=0.9)
    plain = product.options(precision=A.PREC_MIXED, **POLISH)
    train = _vdd_family(nl, 2_000_000, 2048)
    ptrain, _, _ = _dc_batch(product, ctx, nl, train, plain)
    seeder = product.Seeder(ptrain, width=256, hidden_layers=2, init_seed=5)
    assert seeder.add_dc(ptrain) > 1000
    seeder.train(epochs=20, batch=128, lr=1e-3, shuffle_seed=7)
    held = _vdd_family(nl, 3_000_000, 32)
    prob, v_plain, st_plain = _dc_batch(product, ctx, nl, held, plain)
    prob.set_seeder(seeder)
    v, st = prob.solve_dc(product.options(precision=A.PREC_MIXED, seeded=A.SEED_MLP, **POLISH))
    conv = lambda sts: sum(s["status"] == A.ST_CONVERGED for s in sts)
    assert conv(st) >= conv(st_plain)
    checked = 0
    for i in range(0, held.n, 4):
        v_ref, st_ref = port.solve_dc(nl, held, i, linear_solver=1, **POLISH)
        if st_ref["converged"] and st[i]["status"] == A.ST_CONVERGED:
            assert scaled_err(v[i], v_ref) <= 1.0, (i, scaled_err(v[i], v_ref))
            checked += 1
    assert checked >= 4
    assert np.mean([s["iterations"] for s in st]) < np.mean([s["iterations"] for s in st_plain])
    prob.set_seeder(None)
    seeder.close()
