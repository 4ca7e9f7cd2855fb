from .io_ import SetDictionary
