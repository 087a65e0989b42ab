"""Build step of the oracle (test infrastructure).

The oracle of this path is pure numpy (the reference itself is pure Python, so there is
no C/C++ reference source to compile into oracle/_ref); building it is an import check.
"""


def build():
    from . import minres, ssfft_oracle  # noqa: F401
    return True
