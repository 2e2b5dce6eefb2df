"""modisp's CUDA backend plugin, provided by the B200 engine.

modisp imports this package on backend selection and calls ``load()``
(python/modisp/_loader.py:15-28); the returned module implements the plugin
interface over the engine's C ABI.  See modisp_b200/plugin.py.
"""
__version__ = "0.5.0"


def load():
    from modisp_b200 import plugin
    return plugin
