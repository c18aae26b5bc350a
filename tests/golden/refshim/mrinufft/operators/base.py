class FourierOperatorBase:  # pragma: no cover
    def __init__(self, *args, **kwargs):
        raise RuntimeError("mrinufft stub: FourierOperatorBase is not available")
