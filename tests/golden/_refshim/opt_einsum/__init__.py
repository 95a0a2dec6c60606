"""Test-only stand-in for ``opt_einsum`` (pinned 3.4.0 by the reference, ``uv.lock:932-933``).

The reference imports it lazily and only for einsum calls with three or more operands
(``ops/contraction.py:830``).  ``contract_path`` here returns a fixed path -- contract the
first two remaining operands, append the result, repeat -- instead of an optimised one.
The golden vectors that go through it are bosonic (Z2 CTMRG), where every path gives the
same tensor up to rounding; only ``contract_path``'s path output is used by the caller.
"""


def contract_path(equation, *operands, shapes=False, optimize="auto", **kwargs):
    n = len(equation.split("->")[0].split(","))
    return [(0, 1)] * (n - 1), None
