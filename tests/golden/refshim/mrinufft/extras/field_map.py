def __getattr__(name):  # pragma: no cover
    raise RuntimeError(f"mrinufft stub: field_map.{name} is not available")
