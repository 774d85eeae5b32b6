"""``jax.scipy.sparse`` stand-in.  Test infrastructure only."""
from . import linalg  # noqa: F401
