"""Physics and runtime constants (src/physics/constants.ts:11-125)."""

NW = 33.4                                        # molecules / nm^3
BIND = (10.79, 13.39, 16.05, 32.30, 539.0)       # ionisation shells (eV)
EXC_E = (8.22, 10.0, 11.24, 12.61, 13.77)        # excitation levels (eV)
VIB_LEV = (0.01, 0.024, 0.061, 0.092, 0.204, 0.417, 0.460, 0.500, 0.835)
DIFFUSION = {"OH": 2.2, "eaq": 4.9, "H": 7.0, "H3O": 9.0}   # nm^2/ns
SPECIES = {"OH": 0, "eaq": 1, "H": 2, "H3O": 3, "OHminus": 6, "H2": 7}
SOLVATION_THRESHOLD = 7.4

MAX_SEC = 5_000_000
MAX_RAD = 16_000_000
CHEM_N = 8_000_000
VC = 128
HASH_SIZE = 8_388_608
MAX_SEC_STEPS = 2000
MAX_PRIMARY_STEPS = 65536                        # P.ms, dispatch.ts:28

# [speciesA, speciesB, R_nm, pc, product] (constants.ts:313-321)
IRT_REACTIONS = (
    (0, 0, 0.44, 0.376, 1),
    (0, 1, 0.57, 0.980, 0),
    (0, 2, 0.45, 0.511, 0),
    (1, 1, 0.54, 0.125, 2),
    (1, 2, 0.61, 0.455, 2),
    (1, 3, 0.47, 0.538, 3),
    (2, 2, 0.34, 0.216, 2),
)
IRT_D = (DIFFUSION["OH"], DIFFUSION["eaq"], DIFFUSION["H"], DIFFUSION["H3O"])
IRT_RXN_ONSAGER = (
    (0, 0, 0.44, 0, 1),
    (0, 1, 0.57, 0, 0),
    (0, 2, 0.45, 0, 0),
    (1, 1, 0.54, 0, 2),
    (1, 2, 0.61, 0, 2),
    (1, 3, 0.47, 0.71, 3),
    (2, 2, 0.34, 0, 2),
)

KARAMITROS_2011 = {"G_OH": 2.50, "G_eaq": 2.50, "G_H": 0.57, "G_H2O2": 0.73, "G_H2": 0.42}

DNA_LENGTH_NM = 3000
DNA_GRID_N = 21
DNA_SPACING_NM = 150

SSB_R_DAMAGE_NM = 0.29
SSB_P_INDIRECT = 0.4
SSB_P_DIRECT = 0.15
DSB_WINDOW_BP = 10

# The worker's 9-reaction table (public/irt-worker.js:216-226) and its labels
IRT_WORKER_RXN_LABELS = (
    "OH+OH→H2O2 [PDC]", "eaq+OH→OH- [PDC]", "OH+H→H2O [PDC]",
    "eaq+eaq→2OH-+H2 [TDC]", "eaq+H→OH-+H2 [TDC]", "eaq+H3O+→H [PDC]",
    "H+H→H2 [TDC]", "eaq+H2O2→OH-+OH [PDC]", "H3O++OH-→H2O [TDC]",
)
CHECKPOINTS_NS = (0.001, 0.01, 0.1, 1, 10, 100, 1000)
CHECKPOINT_LABELS = ("1 ps", "10 ps", "100 ps", "1 ns", "10 ns", "100 ns", "1 us")

DEFAULT_CHEM_BACKEND = "worker"                  # src/chemistry/backend.ts:18
CHEM_BACKENDS = ("gpu", "worker", "none")
