"""exfemus_b200 -- B200-native element assembly + geometric multigrid for exFEMuS.

The CUDA library (libexfemus_b200.so, built from csrc/ for sm_100a) is the product;
this package loads it through its C ABI and mirrors the reference's MGSolBase
interface.  Importing never falls back to a CPU path: if the library is missing the
first call raises.
"""
from . import _lib  # noqa: F401
from ._lib import ExfError, load  # noqa: F401
from .mgsolver import MGSolBase, MGSolDS, MGSolNS, MGSolT, MGSolTBK, Mesh, mg_params, phys, timestep_loop  # noqa: F401
from .soln_out import print_case, print_soln, read_xdmf, write_xdmf  # noqa: F401
from .workloads import WORKLOADS, make_case  # noqa: F401
