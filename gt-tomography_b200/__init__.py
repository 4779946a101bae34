"""B200-native cone-beam projector and ordered-subset reconstruction core.

A drop-in for the circular-orbit cone-beam path of gt-tomography
(xray/conebeam_projection.cu and the operators/solvers above it).  The
compute lives in libcbct.so (hand-written sm_100a CUDA behind the C ABI of
include/cbct.h); this package is a thin Python view of that ABI shaped like
the reference's operator classes.

The directory name contains a hyphen, so it is imported by path:

    import importlib.util, sys
    spec = importlib.util.spec_from_file_location(
        "gt_tomography_b200", "gt-tomography_b200/__init__.py",
        submodule_search_locations=["gt-tomography_b200"])
    gtb = importlib.util.module_from_spec(spec); sys.modules[spec.name] = gtb
    spec.loader.exec_module(gtb)
"""
from . import _lib  # noqa: F401
from ._lib import CBCT_BF16, CBCT_F16, CBCT_F32, CbctError, lib  # noqa: F401
from . import serving  # noqa: F401
from .serving import Server  # noqa: F401
from .operators import (  # noqa: F401
    CBCT_acquisition, CBCT_binning, CBCT_geometry, CBSubsetOperator, CBSubsetWeightOperator, Plan, batch_osmom,
    cuConebeamProjectionOperator, cuTVPrimalDualOperator,
    default_frequency_filter, fdk_reconstruct_3d, hann_ramp_filter, hoCuConebeamProjectionOperator,
    osMOMSolverD, osSARTSolver, phantom_voxelize, reduce_f64, subset_partition)
from . import phantom  # noqa: F401
from . import acquisition_io  # noqa: F401
from .acquisition_io import read_real, save_real  # noqa: F401

__version__ = "0.1.0"


def build(force: bool = False) -> str:
    """Compiles libcbct.so in-tree for sm_100a (see build.py)."""
    import importlib.util
    import os
    here = os.path.dirname(os.path.abspath(__file__))
    spec = importlib.util.spec_from_file_location("_gtb_build", os.path.join(here, "build.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.build(force=force)
