"""Every threshold the assembly reads, with mhs's values.

Each algorithm constant here changes results, so each equals the value mhs
uses (mhs/defaults.py:23-143, mhs/fullspace/defaults.py:20-35); the device
engine carries the same numbers in ``csrc/engine_base.cuh`` (namespace
``cst``) and a CPU test asserts the two agree.

``MATRIX_MAX_BYTES`` is the one user-facing value: a caller may rebind it to
move the output ceiling.
"""

# output ceiling (mhs/defaults.py:23-26)
MATRIX_MAX_BYTES = 8 * 1024**3
MATRIX_RAM_FRACTION = 0.5
#: Fraction of the device's free memory a device-resident output may take.
MATRIX_DEVICE_FRACTION = 0.9

# near/far split and far-field rules (mhs/fullspace/defaults.py:20-23)
D_STAR = 10.0
FAR_GAUSS_N = 12
FAR_GAUSS_N_DISTANT = 8
D_STAR_DISTANT = 40.0

# edge primitive regimes (mhs/fullspace/defaults.py:30-35)
SERIES_U_OVER_RHO = 2.0
SERIES_TERMS = 32
SMALL_U_OVER_RHO = 0.5
DEGENERATE_AREA_REL = 1e-14

# image Q-family order law (mhs/defaults.py:60-68)
IMAGE_Q_BUDGET_C = 10.0
IMAGE_Q_GAUSS_MIN = 8
IMAGE_Q_GAUSS_MAX = 192

# continuous layout weld (mhs/defaults.py:88)
WELD_TOL_OVER_H = 1.0e-9

# the fold (mhs/defaults.py:108-143)
FOLD_SOURCE_DEPTH_EPS = 3.0
FOLD_BAND_DEPTH_EPS = 10.0
FOLD_REACH_EPS = 60.0
FOLD_N_RADIAL = 6
FOLD_N_ANGULAR = 4
FOLD_CREASE_MARGIN_EPS = 5.0
FOLD_FINE_SPACING_EPS = 0.25
FOLD_MEDIUM_SPACING_EPS = 2.0
FOLD_N_COARSE = 24
FOLD_FINE_SUBPANEL_EPS = 6.0
FOLD_MEDIUM_SUBPANEL_EPS = 16.0
FOLD_R1_MARGIN_DIAM = 8.0

# float32 storage parity (mhs/defaults.py:43)
OUT_FLOAT32_PARITY = 1.0e-6
