"""The runtime options the library reads (option("name", default) in its C++
and CUDA sources) and the option list documented beside
hodlr_b200_set_option in include/hmat_lib/hodlr_b200.h name the same set, so
a new or renamed option cannot go undocumented."""
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
    with open(os.path.join(ROOT, "include", "hmat_lib", "hodlr_b200.h")) as fh:
        text = fh.read()
    block = text.split("Every option the library reads", 1)[1]
    block = block.split("*/", 1)[0]
    # entries: "name (default)" at the start of a documentation line or after
    # a comma inside it
    return set(re.findall(r"(?:^ \*   |, )([a-z][a-z_0-9]+) \(", block, flags=re.M))


def test_every_option_is_documented_and_exists():
    src, doc = _source_options(), _documented_options()
    assert src, "no options found in the sources"
    assert src - doc == set(), f"undocumented options: {sorted(src - doc)}"
    assert doc - src == set(), f"documented options the library does not read: {sorted(doc - src)}"
