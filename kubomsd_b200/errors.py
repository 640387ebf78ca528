"""Error types of the stochastic backend.

When KuboMSD itself is importable its own classes are reused, so a failure
raised by this backend is the very `NumericalError` the reference's callers
catch (src/kubo_msd/errors.py:1-8); otherwise classes with the same names and
hierarchy are defined here.
"""
try:  # pragma: no cover - depends on the host environment
    from kubo_msd.errors import BackendUnavailable, KuboMSDError, NumericalError  # type: ignore
except Exception:  # noqa: BLE001
    class KuboMSDError(ValueError):
        """Invalid input or failed numerical acceptance; never silently repaired."""

    class BackendUnavailable(KuboMSDError):
        pass

    class NumericalError(KuboMSDError):
        pass

__all__ = ["KuboMSDError", "BackendUnavailable", "NumericalError"]
