"""The solver selection mirrors the reference's RiemannSolverFactory
(src/riemann/RiemannSolverFactory.hpp:66-134): "Exact" and "HLLC" by name,
"EXAC" and "HLLC" by restart tag; the reference's other solvers (TRRS,
NoPressure, Advection) are refused as unsupported; an unknown name is an
error, as the reference's my_exit() is."""
import pytest

from shadowfax_b200 import _lib as L
from shadowfax_b200.hydro import (ExactRiemannSolver, HLLCRiemannSolver,
                                  RiemannSolverFactory)


def test_names_and_tags():
    e = RiemannSolverFactory.generate("Exact", 1.4, 1e-6, -2.0)
    assert isinstance(e, ExactRiemannSolver) and e.tag() == "EXAC"
    assert (e.get_gamma(), e.tolerance, e.cutoff, e.kind) == (1.4, 1e-6, -2.0, L.SOLVER_EXACT)
    h = RiemannSolverFactory.generate("HLLC", 1.4)
    assert isinstance(h, HLLCRiemannSolver) and h.tag() == "HLLC" and h.kind == L.SOLVER_HLLC
    d = RiemannSolverFactory.generate("Exact")
    assert (d.get_gamma(), d.tolerance, d.cutoff) == (5 / 3, 1e-8, -5.0)
    assert isinstance(RiemannSolverFactory.from_tag("EXAC"), ExactRiemannSolver)
    assert isinstance(RiemannSolverFactory.from_tag("HLLC"), HLLCRiemannSolver)


@pytest.mark.parametrize("name", ["TRRS", "NoPressure", "Advection"])
def test_other_reference_solvers_are_unsupported(name):
    with pytest.raises(L.SfxError) as e:
        RiemannSolverFactory.generate(name)
    assert e.value.status == L.SFX_ERR_UNSUPPORTED


@pytest.mark.parametrize("tag", ["TRRS", "ADVE", "NOPR"])
def test_other_reference_tags_are_unsupported(tag):
    with pytest.raises(L.SfxError) as e:
        RiemannSolverFactory.from_tag(tag)
    assert e.value.status == L.SFX_ERR_UNSUPPORTED


def test_unknown_name_is_an_error():
    with pytest.raises(ValueError):
        RiemannSolverFactory.generate("Roe")
