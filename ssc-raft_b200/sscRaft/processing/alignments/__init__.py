from .rotationaxis import *  # noqa: F401,F403
