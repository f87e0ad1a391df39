"""The committed ncu summaries: every one names the command that made it (ncu with
--clock-control none, one kernel, one launch) and one traffic figure, and bench.py finds the
traffic of every format it reports."""
import glob
import importlib.util
import os
import re

from conftest import ROOT

PROFILES = sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md")))


def test_every_summary_names_its_command_and_traffic():
    assert len(PROFILES) >= 9
    for p in PROFILES:
        text = open(p).read()
        cmds = [l for l in text.splitlines() if "ncu " in l and ("--set full" in l or "--metrics" in l)]
        assert cmds, p
        for c in cmds:
            assert "--clock-control none" in c, (p, c)
            if "--set full" in c:
                assert "-k regex:" in c and "-c 1" in c, (p, c)
        t = re.findall(r"^traffic_bytes_per_launch: (\d+)$", text, re.M)
        assert len(t) == 1 and int(t[0]) > 0, p


def test_bench_reads_the_traffic_of_every_format():
    spec = importlib.util.spec_from_file_location("bench_mod", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    for fmt in bench.FORMATS + ["csr_f32_dot2"]:
        assert bench.ncu_traffic(fmt) > 0, fmt
