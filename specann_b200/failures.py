"""Exceptions of the solvers, with the same names and meaning as the reference's
(utils/failures.py:4-25, models/spectral_annealing.py:70-77), and its out-of-memory test."""


class NumericalFailure(RuntimeError):
    """The solver ran but produced no valid solution (e.g. the eigensolver failed at every alpha)."""


class EigensolverBreakdown(RuntimeError):
    """The eigensolver produced an unusable result (Lanczos breakdown, non-finite or impossible pair)."""


class SpecAnnOutOfMemory(MemoryError):
    """A device workspace could not be allocated or was too small."""


_OUT_OF_MEMORY_TEXT = ('cuda out of memory', 'cudaerrormemoryallocation', 'out of memory on device',
                       'outofmemoryerror', 'out of memory', 'unable to allocate', 'cannot allocate memory',
                       'bad_alloc', 'out of space', 'memoryerror')


def is_out_of_memory(exc: BaseException) -> bool:
    """True if the exception or one in its cause chain means the host or the GPU ran out of memory."""
    seen = set()
    while exc is not None and id(exc) not in seen and len(seen) < 10:
        seen.add(id(exc))
        if isinstance(exc, MemoryError):
            return True
        if any(s in f"{type(exc).__name__}: {exc}".lower() for s in _OUT_OF_MEMORY_TEXT):
            return True
        exc = exc.__cause__ if exc.__cause__ is not None else exc.__context__
    return False


def is_numerical(exc: BaseException) -> bool:
    """A numerical failure skips one alpha (models/spectral_annealing.py:74-77)."""
    return isinstance(exc, (EigensolverBreakdown, ArithmeticError)) or type(exc).__name__ == "LinAlgError"
