"""Filter configuration selection: analytic FPR, GPU calibration runs, the
exhaustive cost search and the MLP cost model that stands in for it.

The reference's counterpart is src/dtl/filter/model/ (cost_fn.hpp,
optimizer.hpp, skyline_matrix.hpp, calibration.cpp) and
tool/calibration/src/skyline_matrix_builder.cpp.
"""
