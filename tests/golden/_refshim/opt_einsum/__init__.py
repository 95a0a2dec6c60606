"""Test-only stub for ``opt_einsum`` (pinned 3.4.0 by the reference, ``uv.lock:932-933``).

The reference imports it lazily and only for einsum calls with three or more operands
(``ops/contraction.py:830``); no golden vector uses that route, so the stub refuses.
"""


def contract_path(*args, **kwargs):
    raise NotImplementedError("opt_einsum stub: multi-operand einsum paths are not generated")
