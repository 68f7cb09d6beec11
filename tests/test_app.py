"""runValidation (src/app.ts:91-161) on the CUDA path: the 8-energy ESTAR
sweep, chemistry and damage at 10 keV, the results table and JSON."""
import json

import pytest


@pytest.mark.gpu
def test_run_validation_sweep(tmp_path):
    from wgdna import app
    logs = []
    rows = app.run_validation(np=64, boxNm=15000.0, ceEV=7.4, log=lambda m, c="": logs.append(m))
    assert [r["ref"]["E"] for r in rows] == [100, 300, 500, 1000, 3000, 5000, 10000, 20000]
    table = app.results_table(rows)
    assert len(table) == 8
    for t in table:
        assert t["n_therm"] + t["n_esc"] == 64
        assert 0.98 < t["e_conservation"] <= 1.0
        assert t["csda_class"] in ("ok", "meh", "bad")
    ten = rows[6]
    assert ten["result"]["chem_result"] is not None and ten["damage"] is not None
    doc = app.write_results(rows, 64, str(tmp_path / "results.json"))
    back = json.load(open(tmp_path / "results.json"))
    assert back["tenKeV"]["primaryEnergyEv"] == 10000 and len(back["rows"]) == 8
    assert doc["tenKeV"]["chemistry1Us"]["G_OH"] > 0
    assert any("Validation run complete" in m for m in logs)


@pytest.mark.gpu
def test_run_validation_grid_backend_scores_indirect_ssb():
    """With the 'gpu' backend the radical positions reach scoreIndirectSSB
    (app.ts:178-180), unlike the IRT worker, whose SSB_ind stays 0."""
    from wgdna import app
    rows = app.run_validation(np=64, energies=[10000], chemBackend="gpu")
    r = rows[0]
    cr = r["result"]["chem_result"]
    assert cr["timeline"][0]["label"] == "t=0" and len(cr["timeline"]) == 8
    assert cr["chem_pos_final"].size == 4 * cr["chem_n"]
    assert r["damage"] is not None and r["damage"]["ssb_ind"] >= 0
    assert cr["timeline"][-1]["G_OH"] < cr["timeline"][0]["G_OH"]
