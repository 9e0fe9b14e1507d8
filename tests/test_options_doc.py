"""The runtime options the library reads (option("name", default) in its C++
and CUDA sources) and the options table of the integration guide name the
same set, so a new or renamed option cannot go undocumented."""
import os
import re

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _source_options():
    names = set()
    csrc = os.path.join(ROOT, "hmat_lib_b200", "csrc")
    for f in os.listdir(csrc):
        if f.endswith((".cu", ".cpp", ".h", ".cuh")):
            with open(os.path.join(csrc, f)) as fh:
                names |= set(re.findall(r'option\("([a-z_0-9]+)"', fh.read()))
    return names


def _documented_options():
    with open(os.path.join(ROOT, "INTEGRATION.md")) as fh:
        text = fh.read()
    table = text.split("## Runtime options", 1)[1].split("\n## ", 1)[0]
    names = set()
    for line in table.splitlines():
        if line.startswith("| `"):
            first_cell = line.split("|")[1]
            names |= set(re.findall(r"`([a-z_0-9]+)`", first_cell))
    return names


def test_every_option_is_documented_and_exists():
    src, doc = _source_options(), _documented_options()
    assert src, "no options found in the sources"
    assert src - doc == set(), f"undocumented options: {sorted(src - doc)}"
    assert doc - src == set(), f"documented options the library does not read: {sorted(doc - src)}"
