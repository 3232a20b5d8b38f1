"""initialise / reboot, mirroring pyfastflow/flow/environment.py:16-52."""
from .. import constants as cte


def initialise():
    """Mark the environment initialised; raises if already initialised
    (environment.py:28-29).  Kernels here take the grid as runtime arguments,
    so nothing is compiled."""
    if cte.INITIALISED:
        raise RuntimeError("FastFlow already initialized")
    cte.INITIALISED = True


def reboot():
    """Reset the initialised flag (environment.py:42-52)."""
    cte.INITIALISED = False
