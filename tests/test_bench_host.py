"""Host-side logic of bench.py that needs no GPU: fixed launch shapes from --tuning
(with and without the path-kernel threshold), the peak source when the measured-peaks
file is absent, and the argument parser's workloads."""

import sys

import bench


class _FakeCtx:
    def __init__(self):
        self.calls = []

    def set_tuning(self, *args):
        self.calls.append(args)

    def tuning(self):
        return self.calls[-1]

    def autotune(self, probe):
        raise AssertionError("--tuning must not autotune")


def _args(tuning):
    return type("A", (), {"tuning": tuning})()


def test_tuning_with_four_values_keeps_the_default_threshold():
    ctx = _FakeCtx()
    got, source = bench.launch_shapes(_args("64,128,1,4"), ctx, None)
    assert ctx.calls == [(64, 128, 1, 0, 4)]
    assert source == "fixed by --tuning"


def test_tuning_with_five_values_sets_the_path_kernel_threshold():
    ctx = _FakeCtx()
    bench.launch_shapes(_args("256,64,2,8,1073741824"), ctx, None)
    assert ctx.calls == [(256, 64, 2, 0, 8, 1073741824)]


def test_peaks_fall_back_without_the_measured_file(monkeypatch, tmp_path):
    monkeypatch.setattr(bench, "HERE", str(tmp_path))
    hbm, tf, tf_sustained, kind = bench.peaks()
    assert kind == "fallback" and hbm == 6650.0 and tf == 1590.0 and tf_sustained == 1400.0
    (tmp_path / "MEASURED_PEAKS.json").write_text('{"hbm_gbs": 6500, "bf16_tflops": 1600}')
    hbm, tf, tf_sustained, kind = bench.peaks()
    assert kind == "measured" and hbm == 6500.0 and tf == tf_sustained == 1600.0


def test_workloads_are_listed(monkeypatch, capsys):
    monkeypatch.setattr(sys, "argv", ["bench.py", "--help"])
    try:
        bench.main()
    except SystemExit:
        pass
    text = capsys.readouterr().out
    for w in ("thinfilm1080p", "batch32", "film_queries", "configs", "--config-size", "--instanced-spp"):
        assert w in text
