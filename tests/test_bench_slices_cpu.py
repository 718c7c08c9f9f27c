"""bench.py's report of the int8 slice counts: the automatic choices recorded for
the reported workload's own shapes, not those of other shapes the run tuned."""
import importlib.util
import os

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


class _FakeLib:
    def autotune_report(self):
        return {"chi0_i8 slices npr=600 npair~2^18.625 niw=24": 3,
                "chi0_i8 slices npr=600 npair~2^18.625 niw=24 err@2": 0.0129,
                "sigc_i8 slices ngb=600 nm=400 ntq=40 niw=24": 3,
                "sigc_i8 slices ngb=600 nm=400 ntq=40 niw=48": 4,
                "sigc_i8 slices ngb=1500 nm=400 ntq=40 niw=32": 3,
                "sigc_i8 slices ngb=1500 nm=400 ntq=40 niw=32 err@2": 9.8e-4}


def test_slices_of_the_headline_shapes():
    ns = _bench().chosen_slices(_FakeLib(), 0, ("=600 ", "niw=24"))
    assert ns["chi0"] == 3 and ns["sigc"] == 3
    assert ns["products"] == {"chi0": 6, "sigc": 6}
    assert list(ns["estimates"]) == ["chi0_i8 slices npr=600 npair~2^18.625 niw=24 err@2"]


def test_slices_of_the_large_cell_shapes():
    # no chi0 record at N = 1500 (accumulating calls only): the 3 those calls take
    ns = _bench().chosen_slices(_FakeLib(), 0, ("=1500 ",))
    assert ns["chi0"] == 3 and ns["sigc"] == 3
    assert list(ns["estimates"]) == ["sigc_i8 slices ngb=1500 nm=400 ntq=40 niw=32 err@2"]


def test_requested_count_is_reported_as_is():
    ns = _bench().chosen_slices(_FakeLib(), 4)
    assert ns == {"chi0": 4, "sigc": 4, "products": {"chi0": 10, "sigc": 10}}
