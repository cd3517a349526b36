"""The C ABI library loads and exports every symbol include/annie_b200.h
declares; host-only entry points work without a GPU."""
import os
import re

import annie_b200 as A

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for f in sorted(os.listdir(inc)):
        if f.endswith(".h"):
            text = re.sub(r"/\*.*?\*/", "", open(os.path.join(inc, f)).read(), flags=re.S)
            names |= set(re.findall(r"\b(ab_[a-z0-9_]+)\s*\(", text))
    return sorted(names)


def test_header_and_binding_agree():
    names = {n for n, _, _ in A.ABI}
    assert set(declared_symbols()) == names


def test_library_exports_every_declared_symbol():
    L = A.lib(build_if_missing=True)
    for name in declared_symbols():
        assert hasattr(L, name), name


def test_probe_parameter_rule_survey_table():
    # transformGPU.h:822-857 evaluated at the configurations' sizes
    from annie_b200.synth import Xoshiro256ss
    rng = Xoshiro256ss(3)
    assert A.probe(rng.random_odd(262144), 3)[0] == (5, 4, 12, 18)
    assert A.probe(rng.random_odd(2000020), 3)[0] == (5, 4, 15, 17)
    assert A.probe(rng.random_odd(3000000), 3)[0] == (4, 2, 16, 27)


def test_create_without_device_fails_loudly():
    import pytest
    try:
        import torch
        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = os.path.exists("/dev/nvidia0")
    if has_gpu:
        pytest.skip("a GPU is present")
    from helpers import pick_N
    N = pick_N(20000, seed=1)
    with pytest.raises(A.EngineError):
        A.Transform(N, 3)
