"""Host-side helpers of bench.py that need no GPU."""
import importlib.util
import os
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent


def _bench():
    spec = importlib.util.spec_from_file_location("bench_mod", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _FakeHandle:
    """Records one-column products the way saige_grm_get_stats counts them: device ms per
    product (4.0 with the dense flag sums, 3.0 with the missing-call lists) and the
    products that used the lists."""

    def __init__(self):
        self.profiling = []
        self.reset_stats()

    def set_profiling(self, on):
        self.profiling.append(bool(on))

    def reset_stats(self):
        self.st = {"sc_ms": 0.0, "sc_launches": 0, "sc_list_launches": 0}

    def mat_vec(self, v):
        assert v.shape == (1, 12)
        lists = os.environ.get("SAIGE_SR_LISTS") != "0"
        self.st["sc_ms"] += 3.0 if lists else 4.0
        self.st["sc_launches"] += 1
        self.st["sc_list_launches"] += int(lists)

    def stats(self):
        return dict(self.st)


def test_single_column_modes_times_both_sums_and_restores_the_environment(monkeypatch):
    b = _bench()
    for prev in (None, "2"):
        if prev is None:
            monkeypatch.delenv("SAIGE_SR_LISTS", raising=False)
        else:
            monkeypatch.setenv("SAIGE_SR_LISTS", prev)
        h = _FakeHandle()
        out = b.single_column_modes(h, 12, reps=3)
        assert out == {"flags_ms": 4.0, "flags_list_products": 0, "lists_ms": 3.0,
                       "lists_list_products": 3, "products": 3}
        assert os.environ.get("SAIGE_SR_LISTS") == prev
        assert h.profiling == [True, False]
