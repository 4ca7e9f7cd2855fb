from .fbp_methods import *
from .radon_methods import *
from .em_methods import *
from .batch_methods import *
