"""The autotuner's header writer: the entries it writes for a sweep's winners — packed and
early-return variants, a row-limited small-table entry — compile, and the launcher's
lookup (mb::tuned_config) returns them for their shapes, the small-table entry first and
only up to its row limit. Host only: the header is compiled with g++."""
import os
import subprocess

import pytest

from mordred_b200 import autotune as AT

RESULTS = [
    {"shape": "Query B form", "key": [0, 4, 0, 1, 0], "gbs": 4850.0,
     "best": {"threads": 768, "items": 8, "stages": 2, "group_mode": 1, "pack": 2, "ms": 0.594}},
    {"shape": "Query A form", "key": [0, 3, 0, 1, 1], "gbs": 4210.0,
     "best": {"threads": 768, "items": 8, "stages": 3, "group_mode": 2, "pack": 3, "ms": 0.456}},
    {"shape": "engine four-table group-by", "key": [0, 4, 2, 1, 0], "gbs": 4480.0,
     "best": {"threads": 512, "items": 8, "stages": 2, "group_mode": 1, "pack": 1, "ms": 0.643}},
    {"shape": "filter-aggregate (q11 form)", "key": [3, 0, -1, 0, 0], "gbs": 7150.0,
     "best": {"threads": 256, "items": 16, "stages": 4, "group_mode": 0, "pack": 0, "ms": 0.268}},
    {"shape": "filter-aggregate, 6 M rows", "key": [3, 0, -1, 0, 0], "max_rows": 16 << 20, "gbs": 5080.0,
     "best": {"threads": 128, "items": 16, "stages": 2, "grid": 0, "group_mode": 0, "ms": 0.0189}},
]

PROBE = r"""
#include <cstdio>
#include "tuned_configs.h"
static void show(const mb::TunedConfig& c) {
  std::printf("%d %d %d %d %d %d\n", c.threads, c.items, c.stages, c.group_mode, c.mirrors, c.pack);
}
int main() {
  show(mb::tuned_config(0, 4, 0, 2, 175, 120000000));   // Query B (CRYSTAL4, 175 groups)
  show(mb::tuned_config(0, 3, 0, 2, 7000, 120000000));  // Query A (7,000 groups: large)
  show(mb::tuned_config(0, 4, 2, 1, 175, 120000000));   // engine four-table group-by
  show(mb::tuned_config(3, 0, 0, 0, 1, 6000000));       // filter-aggregate, small table
  show(mb::tuned_config(3, 0, 0, 0, 1, 120000000));     // filter-aggregate, large table
  show(mb::tuned_config(1, 3, 0, 2, 7000, 120000000));  // no entry: default, L2 group sums
  return 0;
}
"""


def test_written_header_compiles_and_the_launcher_finds_each_entry(tmp_path, monkeypatch):
    header = tmp_path / "tuned_configs.h"
    header.write_text(open(AT.HEADER).read())
    monkeypatch.setattr(AT, "HEADER", str(header))
    monkeypatch.setattr(AT, "JSON", str(tmp_path / "tuned_configs.json"))
    AT.write(RESULTS, "test")
    assert os.path.exists(tmp_path / "tuned_configs.json")
    src = tmp_path / "probe.cpp"
    src.write_text(PROBE)
    exe = tmp_path / "probe"
    build = subprocess.run(["g++", "-std=c++17", "-I", str(tmp_path), str(src), "-o", str(exe)],
                           capture_output=True, text=True)
    assert build.returncode == 0, build.stderr
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    rows = [tuple(int(x) for x in line.split()) for line in out if line.strip()]
    assert rows[0] == (768, 8, 2, 1, 0, 2)   # packed, early stage return
    assert rows[1] == (768, 8, 3, 2, 0, 3)   # unpacked, early stage return
    assert rows[2] == (512, 8, 2, 1, 0, 1)   # packed
    assert rows[3] == (128, 16, 2, 0, 0, 0)  # the row-limited entry, looked up first
    assert rows[4] == (256, 16, 4, 0, 0, 0)  # past its row limit: the general entry
    assert rows[5] == (256, 8, 2, 2, 0, 0)   # unknown shape with a large group array


@pytest.mark.parametrize("pack", [0, 1, 2, 3])
def test_pack_field_is_written_only_when_set(tmp_path, monkeypatch, pack):
    header = tmp_path / "tuned_configs.h"
    header.write_text(open(AT.HEADER).read())
    monkeypatch.setattr(AT, "HEADER", str(header))
    monkeypatch.setattr(AT, "JSON", str(tmp_path / "tuned_configs.json"))
    r = dict(RESULTS[0], best=dict(RESULTS[0]["best"], pack=pack))
    AT.write([r], "test")
    line = [ln for ln in header.read_text().splitlines() if "Query B form" in ln][0]
    assert ("{768, 8, 2, 1, 0, %d}" % pack in line) if pack else ("{768, 8, 2, 1}" in line)
