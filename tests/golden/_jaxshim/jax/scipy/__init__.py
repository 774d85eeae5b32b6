"""``jax.scipy`` stand-in.  Test infrastructure only."""
from . import sparse  # noqa: F401
