"""Drop-in processes with the reference's module API: each exposes
initialize(cfg, state), update(cfg, state), finalize(cfg, state)
(igm/common/runner/modules/validator.py:1-9).  Install one in place of the
reference's by exposing it as ``iceflow.py`` / ``thk.py`` in the experiment
folder, which the reference's loader imports before its built-ins
(igm/common/runner/modules/loader.py:129-176)."""

from . import iceflow, smb_simple, thk, time, vert_flow  # noqa: F401
