"""IVCurve / IVCurveSolar (LangmuirPython/langmuir/ivcurve.py:15-160,
314-495) restated in langmuir_b200.analysis, on curves with known answers,
and the batched-kMC IV sweep that feeds it (GPU)."""
import numpy as np
import pytest

from langmuir_b200.analysis import IVCurve, IVCurveSolar


def test_units_and_power():
    iv = IVCurve([2.0, -1.0], [0.5, 1.0], 4.0)
    np.testing.assert_allclose(iv.p, [1.0, -1.0])              # nW
    np.testing.assert_allclose(iv.j, [0.5e8, -0.25e8])         # 1 nA/nm^2 = 1e8 mA/cm^2
    np.testing.assert_allclose(iv.r, [0.25e8, -0.25e8])        # 1 nW/nm^2 = 1e8 mW/cm^2
    s = iv.summary()
    assert s["i.max"] == 2.0 and s["i.rng"] == 3.0 and s["a.avg"] == 4.0


@pytest.mark.parametrize("mode,kw", [("interp1d", {}), ("interp1d", {"kind": "linear"}),
                                     ("spline", {}), ("power", {"order": 3})])
def test_linear_cell_has_fill_factor_25(mode, kw):
    # i = k (v + shift - voc): v_oc = voc, i_sc = -k voc, p minimal at voc / 2
    k, voc = 2.0, 0.9
    v = np.linspace(-1.5, 0.5, 21)
    iv = IVCurveSolar(k * (v + 1.5 - voc), v, 1000.0).calculate(mode=mode, **kw)
    assert iv.v_oc == pytest.approx(voc, abs=1e-9)
    assert iv.i_sc == pytest.approx(-k * voc, abs=1e-9)
    # piecewise-linear p(v) has its kinks on the 0.1 V grid: BFGS (gtol 1e-2)
    # stops near, not at, the vertex
    tol = 0.01 if kw.get("kind") == "linear" else 1e-3
    assert iv.v_mp == pytest.approx(voc / 2, abs=tol)
    assert iv.fill == pytest.approx(25.0, abs=100 * tol)
    assert iv.j_sc == pytest.approx(iv.i_sc / 1000.0 * 1e8)
    assert set(("v_oc", "fill", "r_mp")) <= set(iv.summary())


def test_diode_cell_fill_factor_matches_dense_grid():
    n, voc, isc = 0.08, 0.9, -3.0
    f = lambda x: isc * (1 - np.exp((x - voc) / n)) / (1 - np.exp(-voc / n))
    v = np.linspace(-1.5, 0.5, 41)
    iv = IVCurveSolar(f(v + 1.5), v, 1.0).calculate()
    vv = np.linspace(0, voc, 200001)
    exact = (f(vv) * vv).min() / (voc * isc) * 100
    assert iv.v_oc == pytest.approx(voc, abs=1e-3)
    assert iv.fill == pytest.approx(exact, abs=0.2)


def test_unknown_mode():
    with pytest.raises(NotImplementedError):
        IVCurveSolar([1.0, 2.0, 3.0, 4.0], [0.0, 1.0, 2.0, 3.0], 1.0).calculate(mode="cubic")


@pytest.mark.gpu
def test_iv_sweep_on_a_morphology():
    from langmuir_b200 import surrogate as S
    from langmuir_b200.analysis import iv_sweep
    ph, _, _ = S.grf_morphologies(1, size=64, seed=3)
    p = S.solar_label_params(size=64, seed=5, generation=0.2)
    volts = [-1.5, -1.0, -0.5, 0.0, 0.5]
    iv, cur = iv_sweep(p, ph[0].cpu().numpy().reshape(-1), volts, steps=6000, burn_in=1000)
    assert cur.shape == (5,) and np.all(np.isfinite(cur))
    assert cur[0] < cur[-1]                    # the applied field drives the current
    assert np.isfinite(iv.i_sc) and iv.i_sc < 0
