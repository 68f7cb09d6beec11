#!/usr/bin/env python3
"""Extract the reference's own published outputs for this path into
``reference_outputs.json`` (a committed fixture; the tests never read the
reference checkout).

Sources (paths inside the reference checkout):
  validation/webgpu-results.json:1-31                     10 keV, 4096 primaries, box +-15 um, cutoff 7.4 eV
  experiments/results/2026-05-07/level-4/E10-irt-vs-karamitros.json
                                                          summary.perEnergyHeadline: IRT G(1 us) at 1..20 keV
  tests/fixtures/geant4-reference.json                    Geant4-DNA 10 keV figures the reference compares to

Usage:  python make_golden.py <reference checkout>   (or set WGDNA_REFERENCE)
"""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def main(ref):
    web = json.load(open(os.path.join(ref, "validation", "webgpu-results.json")))
    e10 = json.load(open(os.path.join(ref, "experiments", "results", "2026-05-07", "level-4",
                                      "E10-irt-vs-karamitros.json")))
    g4 = json.load(open(os.path.join(ref, "tests", "fixtures", "geant4-reference.json")))
    out = {
        "source": {
            "webgpu_results": "validation/webgpu-results.json",
            "e10": "experiments/results/2026-05-07/level-4/E10-irt-vs-karamitros.json summary.perEnergyHeadline",
            "geant4": "tests/fixtures/geant4-reference.json",
        },
        "webgpu_10keV": {
            "n_primaries": web["nPrimaries"], "E_eV": web["primaryEnergyEv"],
            "tracking": web["tracking"], "pre_chemistry": web["preChemistry"],
            "chemistry_1us": web["chemistry1Us"],
            "dna_damage": {k: v for k, v in web["dnaDamage"].items() if not k.startswith("$")},
        },
        "e10_irt_G_1us": [{"E_eV": r["eEv"], "elapsed_s": r["elapsedSec"], "G": r["g"]}
                          for r in e10["summary"]["perEnergyHeadline"]],
        "e10_meta": {"n_primaries": 4096, "worker": e10["meta"]["sources"]["worker"],
                     "seed": e10["meta"]["seed"]},
        "geant4_10keV": {"track_structure": g4["track_structure"],
                         "chemistry_timeline": g4["chemistry_timeline"]["checkpoints"],
                         "karamitros_2011_1us": {k: v for k, v in g4["karamitros_2011"].items() if k != "note"}},
    }
    with open(os.path.join(HERE, "reference_outputs.json"), "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
        f.write("\n")


if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("WGDNA_REFERENCE")
    if not ref:
        sys.exit("usage: make_golden.py <reference checkout> (or set WGDNA_REFERENCE)")
    main(ref)
