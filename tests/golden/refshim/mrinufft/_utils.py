def proper_trajectory(*args, **kwargs):  # pragma: no cover
    raise RuntimeError("mrinufft stub: proper_trajectory is not available")
