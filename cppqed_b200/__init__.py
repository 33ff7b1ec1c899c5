"""cppqed_b200 — a B200 Monte Carlo wave-function ensemble engine with C++QED's
operator interface (Tridiagonal terms on tensor-product axes, jump operators,
linear averages).  The engine is the shared library built by
:mod:`cppqed_b200.build`; this package is the Python view of its C ABI."""
from .engine import EngineError, Ensemble, Master, Model, Server, System, device_count, lib, mcwf_pars  # noqa: F401
from .evolve import evolve  # noqa: F401
