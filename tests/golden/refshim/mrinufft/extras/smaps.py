def coil_compression(*args, **kwargs):  # pragma: no cover
    raise RuntimeError("mrinufft stub: coil_compression is not available")
