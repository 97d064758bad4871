"""bench.py's bookkeeping on the CPU: the DRAM traffic record is parsed from
an ncu --csv metrics log, keyed by the kernel sources' sha256, and reported
only while the sources are unchanged; both arms print the same config; the
reference arm's steps are bounded samples whose time is the step time."""
import importlib.util
import json
import os

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture()
def bench(tmp_path, monkeypatch):
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    monkeypatch.setattr(mod, "TRAFFIC_RECORD", str(tmp_path / "ncu_traffic.json"))
    return mod


def _csv(tmp_path, rows):
    head = ('"ID","Process ID","Process Name","Host Name","Kernel Name","Context","Stream","Block Size",'
            '"Grid Size","Device","CC","Section Name","Metric Name","Metric Unit","Metric Value"\n')
    lines = ["==PROF== noise line\n", head]
    for i, (kern, metric, unit, val) in enumerate(rows):
        lines.append(f'"{i // 2}","1","python","h","{kern}","1","7","(256, 1, 1)","(9, 1, 1)","0","10.0",'
                     f'"Command line profiler metrics","{metric}","{unit}","{val}"\n')
    p = tmp_path / "dram.csv"
    p.write_text("".join(lines))
    return str(p)


def test_traffic_record_roundtrip(bench, tmp_path):
    fwd = "void viss::k_forward<256, 4, 2, 1, 0>(viss::FwdParams)"   # as ncu names it
    adj = "void viss::k_adjoint<128, 8, 4, 1, 0, 0>(viss::AdjParams)"
    rows = []
    for mb in (90, 100, 101, 102):             # four launches of one forward instance
        rows += [(fwd, "dram__bytes_read.sum", "Mbyte", f"{mb}"), (fwd, "dram__bytes_write.sum", "byte", "1,000")]
    rows += [(adj, "dram__bytes_read.sum", "Gbyte", "0.5"), (adj, "dram__bytes_write.sum", "Mbyte", "2")]
    form = "void viss::k_form_forward<10>(viss::FormParams)"
    rows += [(form, "dram__bytes_read.sum", "Mbyte", "33"), (form, "dram__bytes_write.sum", "byte", "0")]
    rec = bench.record_traffic(_csv(tmp_path, rows), "c3_10mhz", "ncu ...")
    got = rec["bytes_per_launch"]["c3_10mhz"]
    assert got["k_forward<256, 4, 2, 1, 0>"] == 100_501_000      # median of four launches
    assert got["k_adjoint<128, 8, 4, 1, 0, 0>"] == 502_000_000
    assert got["k_form_forward<10>"] == 33_000_000
    v, src = bench.measured_traffic("c3_10mhz", bench.FWD_INSTANCES[0].format(m=1))
    assert v == 100_501_000 and "these kernel sources" in src and "ncu ..." in src
    assert bench.measured_traffic("c3_10mhz", bench.FWD_INSTANCES[1].format(m=1))[0] is None
    assert bench.measured_traffic("c2", "k_forward<256, 4, 2, 1, 0>")[0] is None
    # a record of other kernel sources is never reported
    d = json.loads(open(bench.TRAFFIC_RECORD).read())
    d["kernel_sources_sha256"] = "0" * 64
    open(bench.TRAFFIC_RECORD, "w").write(json.dumps(d))
    v, src = bench.measured_traffic("c3_10mhz", "k_forward<256, 4, 2, 1, 0>")
    assert v is None and "other kernel sources" in src


def test_both_arms_print_the_same_config(bench):
    class A:
        workload = "c3_10mhz"
        formation = False
    c = bench.bench_config(A, 786432, 388800, 1)
    assert c == bench.bench_config(A, 786432, 388800, 1)
    assert c["terms_per_step"] == 2 * 786432 * 388800
    assert set(c) == {"workload", "pixels", "samples", "terms_per_step", "l2", "parallelism"}


def test_reference_arm_steps_are_bounded_samples(bench):
    import argparse
    args = argparse.Namespace(workload="c1", steps=2, warmup=1, cpu_seconds=2.0, reference_seconds=3.0,
                              formation=False)
    r = bench.run_reference(args, 0, 1)
    assert r["impl"] == "reference" and r["steps"] == 2
    # the driver checks ms_per_step x steps against its own clock: one sample per step
    assert r["ms_per_step"] * r["steps"] / 1e3 < 30
    assert r["config"] == bench.bench_config(args, 12288, 10080, 1)
    assert r["cpu_baseline"]["kind"] == "port" and r["e2e"]["h2d_bytes_per_step"] == 0
    assert bench.run_reference(args, 1, 2) is None      # only rank 0 prints


def test_workloads_and_traffic_key(bench):
    """Every workload name resolves to a configuration (the profiling-size
    gridded case: Nside 256 x 48,600 samples at 1 MHz); the traffic record is
    keyed on the measured kernels' translation units only, so a change to
    another source (the gridded adjoint's) leaves it valid."""
    for name in bench.WORKLOAD_TEXT:
        if name in ("c4", "c5", "stream"):
            continue
        cfg = bench.workload_config(name)
        assert cfg.nside > 0 and cfg.n_samples > 0, name
    small = bench.workload_config("c3_small_1mhz")
    assert (small.nside, small.n_samples, small.freqs_hz) == (256, 48600, (1e6,))
    assert "gridded.cu" not in bench.TRAFFIC_KERNEL_SOURCES
    assert {"visibility.cu", "formation.cu"} <= set(bench.TRAFFIC_KERNEL_SOURCES)
    a = bench.kernel_sources_sha()
    assert a == bench.kernel_sources_sha() and len(a) == 64
