"""sscRaft (B200 build): drop-in for the parallel-beam reconstruction hot path
of cnpem/ssc-raft -- fbp (RT), em (tEMRT, eEMRT), radon_RT, lowpass and the
flat/dark correction (correct_projections, correct_background) --
backed by hand-written sm_100a kernels in lib/libraft.so."""
__version__ = "0.1.0+b200"

from .rafttypes import CNICE, FilterNumber, libraft, logger, setInterpolation  # noqa: F401
from .io import SetDictionary  # noqa: F401
from .geometries import *  # noqa: F401,F403
from .geometries.methods import fbp, em  # noqa: F401
from .processing import lowpass, correct_projections, correct_background  # noqa: F401
