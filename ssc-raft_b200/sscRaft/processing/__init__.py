from .filters import *  # noqa: F401,F403
from .background_correction import *  # noqa: F401,F403
from .background_correction import _background_correctionGPU  # noqa: F401
from .alignments import *  # noqa: F401,F403
