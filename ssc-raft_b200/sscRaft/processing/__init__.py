from .filters import *
