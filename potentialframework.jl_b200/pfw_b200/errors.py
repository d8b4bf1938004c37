"""Exceptions of the host mirror, named after the reference's Julia errors.

Every library status maps to one of them (ArgumentError ↔ PFW_EINVAL,
DomainError ↔ PFW_EDOMAIN, DimensionMismatch ↔ PFW_ESHAPE); the model
readers raise the same classes as the reference's readers
(ACE/resolved.jl:57-142, ACE/persistence.jl:25-52).
"""

OK, EINVAL, EDOMAIN, ESHAPE, ECAPACITY, ECUDA, ETIMEDOUT, ESTATE = range(8)


class PFWError(RuntimeError):
    """Error status from the library; subclasses mirror the reference's exceptions."""

    def __init__(self, code, msg):
        super().__init__(msg)
        self.code = code


class ArgumentError(PFWError, ValueError):
    pass


class DomainError(PFWError, ArithmeticError):
    pass


class DimensionMismatch(PFWError, ValueError):
    pass


def argument_error(msg):
    return ArgumentError(EINVAL, msg)


def dimension_mismatch(msg):
    return DimensionMismatch(ESHAPE, msg)
