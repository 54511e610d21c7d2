"""Runner of the reference's own Fortran 90 source for the Biot-Savart / RK4 path.

TEST INFRASTRUCTURE ONLY: used by tests/ and by the fixture script
tests/golden/make_reference_fixtures.py to check the C oracle against the
reference's code itself. The product never imports it.

Neither machine has a Fortran compiler, so the reference's modules cannot be
built. This package reads the reference's free-form .f90 sources where they
lie (nothing of them is copied into this repository), parses the subset of
Fortran 90 its hot path uses, and translates each needed procedure to a
Python function that is then executed:

* REAL(8) arithmetic as IEEE binary64 with every operation rounded once, in
  the order the source's parse tree gives (left to right, parentheses kept);
  this is what a compiler does without value-changing optimisations, and what
  the C oracle's strict build (gcc -O2 -ffp-contract=off) does;
* SUM and DOT_PRODUCT as left-to-right loops in array-element order;
  transcendental intrinsics through the C library (Python's math module);
  integer powers by binary powering (GCC's __powidf2); integer division
  truncating toward zero;
* arrays column-major with their declared lower bounds; dummy arguments by
  reference (arrays and derived types shared, scalars written back when the
  dummy may change them); generic interfaces resolved by argument types;
* MPI (`include 'mpif.h'`) supplied by the caller as host procedures, so ranks
  can run as threads with an in-process broadcast.

What falls outside the subset raises FortranSubsetError with file and line:
the runner never guesses. Generated code is kept in memory (and may be
written to oracle/_ref/ for inspection), never committed.
"""
from __future__ import annotations

from . import rt
from .gen import Program
from .lex import FortranSubsetError

__all__ = ["Runner", "FortranSubsetError", "rt"]


class Instance:
    """One independent copy of the program's modules (one MPI rank, say)."""

    def __init__(self, mods, procs, types):
        self.mods = mods
        self.procs = procs
        self.types = types

    def mod(self, name):
        return self.mods[name.lower()]

    def proc(self, module, name):
        return self.procs[(module.lower(), name.lower())]

    def new(self, module, tname):
        return self.types[(module.lower(), tname.lower())]()


class Runner:
    """Parse the given source files and generate the entry points (and all they reach)."""

    def __init__(self, files, entry_points, includes=None, host_procs=(), stubs=None, use_aliases=None):
        self.prog = Program(files, includes=includes, host_procs=host_procs, stubs=stubs,
                            use_aliases=use_aliases)
        self.source = self.prog.generate([(m.lower(), p.lower()) for m, p in entry_points])
        self._build = _compile(self.source, "<fortran-subset>")

    def instance(self, host=None) -> Instance:
        return Instance(*self._build(rt, host or {}))

    def save(self, path, note=""):
        """Write the generated program (for a machine without the Fortran sources: the
        translation is to the sources what a build is, and stays out of version control)."""
        with open(path, "w") as f:
            f.write("# Generated by oracle/f90 from Fortran sources; a build output, not committed.\n")
            if note:
                f.write(f"# {note}\n")
            f.write(self.source)


class Program_:
    """A generated program loaded back from a file written by Runner.save."""

    def __init__(self, path):
        with open(path) as f:
            self.source = f.read()
        self._build = _compile(self.source, str(path))

    def instance(self, host=None) -> Instance:
        return Instance(*self._build(rt, host or {}))


def load(path) -> Program_:
    return Program_(path)


def _compile(source, name):
    ns: dict = {}
    exec(compile(source, name, "exec"), ns)
    return ns["_build"]
