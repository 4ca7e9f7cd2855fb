"""Dictionary defaults (sscRaft/io/io_.py:131-183 of cnpem/ssc-raft); the
HDF5 readers/writers of that module are outside this library's scope."""
from ..rafttypes import logger


def _SetDic(dic, paramname, deff):
    try:
        dic[paramname]
        if type(dic[paramname]) == list:
            for i in range(len(deff)):
                try:
                    dic[paramname][i]
                except Exception:
                    value = deff[i]
                    logger.info(f'Using default {paramname}:{value}')
                    dic[paramname][i] = value
    except Exception:
        logger.info(f'Using default {paramname}: {deff}.')
        dic[paramname] = deff
    return dic


def _EvalRequiredDic(dic, paramname):
    for key in paramname:
        try:
            dic[key]
        except Exception:
            message_error = f'Missing required dictionary key: {key}'
            logger.info(message_error)
            raise ValueError(message_error)
    return dic


def SetDictionary(dic, required, optional, default):
    """Check required keys (ValueError if missing) and fill optional keys
    with defaults, in place."""
    dic = _EvalRequiredDic(dic, required)
    for key in range(len(optional)):
        dic = _SetDic(dic, optional[key], default[key])
    return dic
