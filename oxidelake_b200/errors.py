"""EngineError, mirrored from crates/oxidelake-core/src/error.rs:17-73.

The C ABI returns an ``oxb_status``; the host layer raises the matching
subclass with the library's message.  ``Unsupported`` is the only error a
caller may answer by taking its own CPU path (error.rs:56-64, is_unsupported
:118); every other error fails the query.
"""
from __future__ import annotations


class EngineError(Exception):
    """Base of every error the GPU operator path raises."""

    status = -1

    def is_unsupported(self) -> bool:
        return isinstance(self, Unsupported)


class Unsupported(EngineError):
    status = 1


class Device(EngineError):
    status = 2


class Execution(EngineError):
    status = 3


class Plan(EngineError):
    status = 4


class Allocation(EngineError):
    status = 5


class AdmissionRejected(EngineError):
    """A served request's estimated device memory exceeds the budget."""

    status = 6


class TableFull(EngineError):
    status = 7


class Timeout(EngineError):
    status = 8


_BY_STATUS = {c.status: c for c in (Unsupported, Device, Execution, Plan, Allocation, AdmissionRejected, TableFull, Timeout)}


def error_for(status: int, message: str) -> EngineError:
    return _BY_STATUS.get(status, EngineError)(message)
