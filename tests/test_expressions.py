"""The engine's expression language (the .pro expression subset): parser,
tree evaluation and the compiled register program agree with Python."""
import math

import pytest

from dynlattice_b200.engine import DLError, eval_expression

CASES = [
    ("1 + 2 * 3", {}, 7.0),
    ("2 ^ 3 ^ 2", {}, 2.0 ** 9),
    ("-2 ^ 2", {}, -4.0),
    ("(1 + 2) * 3 - 4 / 8", {}, 8.5),
    ("sqrt(12/2e3)", {}, math.sqrt(12 / 2e3)),
    ("5.6e10/12", {}, 5.6e10 / 12),
    ("if(t<15, 6/15 * (1 - cos(2*PI/15 * t)), 0)", {"t": 3.0}, 6 / 15 * (1 - math.cos(2 * math.pi / 15 * 3.0))),
    ("if(t<15, 6/15 * (1 - cos(2*PI/15 * t)), 0)", {"t": 20.0}, 0.0),
    ("min(i/500, 1)", {"i": 250}, 0.5),
    ("min(i/500, 1)", {"i": 2500}, 1.0),
    ("t % 0.1 < deltaTime", {"t": 0.30001, "deltaTime": 1e-4}, 1.0),
    ("abs(dx) + abs(dy) - 10 * (1 + 0*h_0)", {"dx": -3.0, "dy": 4.0, "h_0": 7.0}, -3.0),
    ("abs(dx/( 700-h_dx))^2.04", {"dx": -300.0, "h_dx": 20.0}, (300 / 680) ** 2.04),
    ("2.04 * abs(dx/(700-h_dx))^1.04 * if(dx/(700-h_dx)>0, 1, if(dx/(700-h_dx)<0, -1, 0)) / (700-h_dx)",
     {"dx": -300.0, "h_dx": 20.0}, 2.04 * (300 / 680) ** 1.04 * -1 / 680),
    ("max(1, 2, 3) + min(4, -5)", {}, -2.0),
    ("sign(-3) + floor(2.7) + ceil(2.1) + exp(0) + log(1) + atan(0) + tan(0) + sin(0)", {}, 5.0),
    ("!(1 > 2) && (3 >= 3) || 0", {}, 1.0),
    ("x == 2 != 0", {"x": 2.0}, 1.0),
    ("pow(2, 10) + .5", {}, 1024.5),
]


@pytest.mark.parametrize("expr,vars,expected", CASES)
def test_expression_values(expr, vars, expected):
    assert eval_expression(expr, **vars) == pytest.approx(expected, rel=1e-14, abs=1e-300)


@pytest.mark.parametrize("bad", ["1 +", "foo + 1", "sqrt(1, 2)", "(1 + 2", "1 $ 2", "if(1, 2)"])
def test_expression_errors(bad):
    with pytest.raises(DLError):
        eval_expression(bad)


def test_yield_expression_of_lattice_material():
    from dynlattice_b200.lattices import aluminium_elastoplastic
    m = aluminium_elastoplastic(radius=0.5e-3)
    r = 0.5e-3
    A = math.pi * r * r
    sy = 300e6
    args = dict(dx=1.0, dy=-2.0, dz=150.0, rx=0.01, ry=-0.02, rz=0.005, h_0=-3.0, radius=r, area=A)
    Np, Vp = sy * A, sy / math.sqrt(3) * A
    Mp, Tp = sy * 4 / 3 * r ** 3, sy / math.sqrt(3) * 2 / 3 * math.pi * r ** 3
    s = math.sqrt((1 / Vp) ** 2 + (2 / Vp) ** 2 + (150 / Np) ** 2 + (0.01 / Mp) ** 2 + (0.02 / Mp) ** 2
                  + (0.005 / Tp) ** 2)
    f = s - 1 + (-3.0) / (sy * math.sqrt(A))
    assert eval_expression(m.yield_cond, **args) == pytest.approx(f, rel=1e-13)
    # yieldDeriv is the analytic gradient of yieldCond (central differences)
    names = ["dx", "dy", "dz", "rx", "ry", "rz", "h_0"]
    for name, d in zip(names, m.yield_deriv):
        h = 1e-6 * max(1.0, abs(args[name]))
        ap = dict(args); ap[name] += h
        am = dict(args); am[name] -= h
        fd = (eval_expression(m.yield_cond, **ap) - eval_expression(m.yield_cond, **am)) / (2 * h)
        assert eval_expression(d, **args) == pytest.approx(fd, rel=1e-6, abs=1e-12)
