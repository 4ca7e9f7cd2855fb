from .parallel import *
from .methods import *
