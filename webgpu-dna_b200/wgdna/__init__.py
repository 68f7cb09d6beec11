"""wgdna -- B200 CUDA path of allaunthefox/webgpu-dna's hot path.

Electron track transport in liquid water -> Karamitros 9-reaction IRT
chemistry -> SSB/DSB scoring on the 21x21 B-DNA fibre grid, behind the
reference's own surface (runValidation, runAtEnergy, runChemistryWorker, the
scoring functions, the tables and the results JSON).  Every call goes through
the C ABI of libwgdna.so (include/wgdna.h); there is no CPU fallback.
"""
from . import constants
from ._lib import Context, WgdnaError, lib, EXPORTS, LIB_PATH, TABLES_PATH
from .app import ensure_pipelines, ensurePipelines, results_json, run_validation, runValidation
from .chemistry import run_chemistry_device, run_chemistry_worker, runChemistryWorker
from .dispatch import aggregate, run_at_energy, runAtEnergy, transport_params
from .estar import ESTAR, find_estar
from .geometry import DNATarget, build_dna_target, buildDNATarget
from .scoring import (SsbRng, cluster_dsb, clusterDSB, combine_hits, combineHits, make_ssb_rng, makeSsbRng,
                      score_direct_ssb_events, score_indirect_ssb, scoreDirectSSB_events, scoreIndirectSSB)

__all__ = [n for n in dir() if not n.startswith("_")]
