"""Import shim for the package directory ``acoustic-agent_b200/``.

The directory name is not a Python identifier, so this module stands in for
it: it turns itself into a package whose ``__path__`` is that directory and
runs the directory's ``__init__.py``.  ``import acoustic_agent_b200`` and
``import acoustic_agent_b200.backend`` then work from the repository root.
"""
import os as _os

__path__ = [_os.path.join(_os.path.dirname(_os.path.abspath(__file__)), "acoustic-agent_b200")]
_init = _os.path.join(__path__[0], "__init__.py")
with open(_init, "r", encoding="utf-8") as _fh:
    exec(compile(_fh.read(), _init, "exec"))
del _fh, _init
