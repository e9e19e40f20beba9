"""GPU float64 flow-field generation against the reference's own generator.

tests/golden/flowgen.npz holds the raw output of the reference's
generate_flow_field (python/gamma_smc_cu/demographic.py:146-208, numpy/scipy)
for a constant-Ne grid and a three-epoch history (script beside it).  Where
the reference's fit is meaningful (finite, |u|, |v| <= 1e3) the GPU result
must agree within 1e-6 relative (absolute floor 1e-9); a handful of cells
with nearly collinear design columns sit near that bound, the rest agree to
~1e-11.  Cells the reference skips are 0 in both; cells where the reference
returns non-finite or huge values (the tiny-mean, tiny-CV corner) must be
non-finite, huge or 0 here too -- those are the cells the fixture file zeroes.
"""
import os

import numpy as np
import pytest

from gamma_smc_cu_b200 import _core, demographic, synthetic

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = np.load(os.path.join(HERE, "golden", "flowgen.npz"))
CASES = {
    "const": {},
    "demo": {"Ne_values": [2.0e4, 5.0e3, 1.5e4], "epoch_boundaries": [0.0, 2.0e3, 3.0e4],
             "Ne_ref": 1.0e4, "n_steps": 200},
}


def _garbage(x):
    return ~np.isfinite(x) | (np.abs(x) > 1e3)


@pytest.mark.parametrize("name", sorted(CASES))
def test_flow_field_matches_reference_generator(name):
    u, v = demographic.generate_flow_field(verbose=False, **CASES[name])
    for got, want in ((u, GOLD[f"{name}_u"]), (v, GOLD[f"{name}_v"])):
        assert got.shape == want.shape == (51, 50)
        valid = ~_garbage(want)
        err = np.abs(got - want)[valid] / np.maximum(np.abs(want[valid]), 1e-3)
        assert err.max() <= 1e-6, err.max()
        assert np.array_equal(got[want == 0], want[want == 0])
        bad = ~valid
        assert (_garbage(got[bad]) | (got[bad] == 0)).all()


def test_generated_field_drives_the_scan(tmp_path, small_data, oracle):
    """The GPU field, sanitised like the fixture and written in the text
    format, decodes within 1e-4 of the fixture (the reference's own field)."""
    u, v = demographic.generate_flow_field(verbose=False)
    bad = _garbage(u) | _garbage(v)
    u, v = np.where(bad, 0.0, u), np.where(bad, 0.0, v)
    path = str(tmp_path / "gpu_field.txt")
    demographic.write_flow_field(path, u, v)
    ru, rv, *bounds = demographic.load_flow_field(path)
    assert np.allclose(ru, u, atol=1e-10) and bounds == [1e-5, 1e2, 1e-2, 1.0]
    G, pos = small_data
    mu, rho = oracle.estimate_scaled_params(G, pos, 1.25e-8, 1e-8, 1e4)
    pairs = synthetic.all_pairs(40)[::9]
    got = _core.FlowContext(G, pos, 1e4, mu, rho, path, 0).run_fb(pairs)["mean"]
    want = _core.FlowContext(G, pos, 1e4, mu, rho, _core.DEFAULT_FLOW_FIELD, 0).run_fb(pairs)["mean"]
    rel = np.abs(got.astype(np.float64) - want) / want
    assert rel.max() <= 1e-4, rel.max()


def test_demographic_context(small_data, flow_field):
    G, pos = small_data
    d = demographic.DemographicFlowContext(G, pos, 1e4, 1.25e-8, 1e-8, flow_field,
                                           n_calibration_pairs=20, n_epochs=6, n_steps=100,
                                           verbose=False)
    ne, edges = d.demography
    assert ne.shape == (6,) and edges.shape == (7,) and (ne >= 100).all()
    r = d.run_fb([(3, 1), (7, 2)])
    assert r["mean"].shape == (G.shape[1], 2) and np.isfinite(r["mean"]).all()
    s = d.run_fb_summary([(3, 1), (7, 2)])
    assert s["site_mean"].shape == (G.shape[1],)
    f = d.run_fwd([(3, 1)])
    assert f["mean"].shape == (G.shape[1], 1)
