"""The frozen flops per Stokes evaluation (oracle/opcount.py).

The counted restatement must compute what the oracle computes (orc_solfund,
after src/Solfund.for:18-60) before its tally means anything; then the tally
is input-independent and equals the figure bench.py divides the assembly's
evaluation rate by.
"""
import math
import os
import sys

import numpy as np
import pytest

import oracle

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "oracle"))
import opcount  # noqa: E402


def _case(rng):
    p = rng.uniform(-5, 5, 3)
    g = p + rng.uniform(-3, 3, 3)
    rn = rng.standard_normal(3)
    rn /= np.linalg.norm(rn)
    ge, rnu, dam, rho = 1.0 + rng.random(), rng.uniform(0.15, 0.35), rng.uniform(0, 0.05), 1.0
    zge = complex(ge, 2.0 * ge * dam)
    zcs = np.sqrt(zge / rho)
    zcp = zcs * math.sqrt((2.0 - 2.0 * rnu) / (1.0 - 2.0 * rnu))
    return p, g, rn, zge, complex(zcs), complex(zcp), rng.uniform(0.1, 10.0)


def _oracle_solfund(p, g, rn, zge, zcs, zcp, fr):
    zu = np.zeros(9, dtype=np.complex128)
    zt = np.zeros(9, dtype=np.complex128)
    f = lambda z: np.array([z.real, z.imag])  # noqa: E731
    oracle.lib().orc_solfund(np.ascontiguousarray(p), np.ascontiguousarray(g), np.ascontiguousarray(rn),
                             f(zge), f(zcs), f(zcp), fr, zu, zt)
    return zu.reshape(3, 3), zt.reshape(3, 3)  # [j][i] == Z(I,J)


def test_counted_restatement_computes_the_oracle_values():
    rng = np.random.default_rng(11)
    for _ in range(40):
        p, g, rn, zge, zcs, zcp, fr = _case(rng)
        zu, zt = opcount.stokes_eval(p, g, rn, zge, zcs, zcp, fr, 1.0)
        mu = np.array([[zu[j][i].value for i in range(3)] for j in range(3)])
        mt = np.array([[zt[j][i].value for i in range(3)] for j in range(3)])
        ou, ot = _oracle_solfund(p, g, rn, zge, zcs, zcp, fr)
        assert np.linalg.norm(mu - ou) <= 1e-13 * np.linalg.norm(ou)
        assert np.linalg.norm(mt - ot) <= 1e-13 * np.linalg.norm(ot)


def test_counted_geometry_is_the_bilinear_map():
    rng = np.random.default_rng(5)
    co = np.array([[0.0, 0.0, 0.0], [1.0, 0.1, 0.0], [1.1, 1.0, 0.05], [-0.1, 0.9, 0.0]])
    co += 0.05 * rng.standard_normal(co.shape)
    for g1, g2 in rng.uniform(-1, 1, (10, 2)):
        x, y, z, det = opcount.gauss_geometry(co.tolist(), g1, g2)
        f = 0.25 * np.array([(1 - g1) * (1 - g2), (1 + g1) * (1 - g2), (1 + g1) * (1 + g2), (1 - g1) * (1 + g2)])
        dg1 = 0.25 * np.array([-(1 - g2), (1 - g2), (1 + g2), -(1 + g2)])
        dg2 = 0.25 * np.array([-(1 - g1), -(1 + g1), (1 + g1), (1 - g1)])
        assert np.allclose([x.v, y.v, z.v], f @ co, atol=1e-14)
        assert det.v == pytest.approx(np.linalg.norm(np.cross(dg1 @ co, dg2 @ co)), rel=1e-13)


def test_counts_are_input_independent_and_frozen():
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    rng = np.random.default_rng(3)
    first = opcount.count_stokes()
    for _ in range(5):
        p, g, rn, zge, zcs, zcp, fr = _case(rng)
        c = opcount.count_stokes(p=tuple(p), g=tuple(g), rn=tuple(rn), zge=zge, zcs=zcs, zcp=zcp,
                                 fr=fr, p12=float(rng.random()))
        assert c == first
    assert first["flops"] == bench.STOKES_FLOPS_PER_EVAL
    assert (first["exp"], first["sincos"]) == (2, 2)
    assert opcount.count_geometry()["flops"] == bench.GEOMETRY_FLOPS_PER_GAUSS_POINT


def test_bench_assembly_roofline_uses_the_frozen_count():
    """bench.py's assembly roofline on a fixed kernel record: evaluations per
    second x the frozen flops against the measured FP64 FMA peak."""
    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    k = {"ms": 30.0, "launches": 3, "work": 1.5e9, "bytes": 2.0e10}
    r = bench._roofline("assembly", k, {"hbm_gbs": 6517.0}, {"fp64_fma": 35.0})
    evals = 1.5e9 / 0.030
    assert r["stokes_evals_per_s"] == pytest.approx(evals)
    assert r["fp64"]["achieved_tflops"] == pytest.approx(evals * 613 / 1e12, abs=0.01)
    assert r["fp64"]["frac"] == pytest.approx(evals * 613 / 1e12 / 35.0, abs=1e-4)
    # without a measured FP64 peak the fraction is left open, not invented
    r = bench._roofline("assembly", k, {"hbm_gbs": 6517.0}, {})
    assert r["fp64"]["frac"] is None
