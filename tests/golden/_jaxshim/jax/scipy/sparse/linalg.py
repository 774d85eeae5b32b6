"""``jax.scipy.sparse.linalg`` stand-in.  Test infrastructure only; the
shimmed production paths never call ``cg`` (column projection is off)."""


def cg(*_args, **_kwargs):  # pragma: no cover
    raise NotImplementedError("cg is not available in the NumPy shim")
