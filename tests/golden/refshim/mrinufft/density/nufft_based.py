def pipe(*args, **kwargs):  # pragma: no cover
    raise RuntimeError("mrinufft stub: pipe density is not available")
