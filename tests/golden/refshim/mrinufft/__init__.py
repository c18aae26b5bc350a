"""Minimal stand-in for the absent ``mrinufft`` package.

Only what importing the reference ``pygrog`` needs.  ``with_torch`` is the
one function on the GROG hot path; it is a container conversion (numpy in ->
torch inside -> numpy out) with no arithmetic.  Everything else raises, so a
reference code path that really needs mrinufft fails loudly.
"""


def get_operator(name):  # pragma: no cover - off the hot path
    raise RuntimeError(f"mrinufft stub: NUFFT backend {name!r} is not available")
