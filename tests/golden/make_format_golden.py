"""Generates the format fixtures (tests/golden/formats_*) with the reference's
own converters and readers.  Run where the reference tree is mounted:

    python tests/golden/make_format_golden.py <reference root>

The fixture graph is R-MAT scale 7 / ef 4 from the product's generator,
stored in the reference's text CSR format (formats_rmat7_rowOffsets.txt,
formats_rmat7_colIndices.txt).  From it:
  formats_rmat7.mtx        scripts/2-datasets/gunrock/csr_to_gunrock_mm.py (convert_to_mtx)
  formats_rmat7.ligra      scripts/2-datasets/ligra/csr_to_ligra_adj.py (convert_to_ligra)
  formats_rmat7_src_nodes.txt
                           scripts/2-datasets/src_nodes/generate_src_lists.py
                           (analyze_graph, 12 samples, Python's random seeded with 5)
  formats_sources_tricky.txt  a hand-written list with comments, blank lines
                           and several ids per line
  formats_*.ids            what scripts/4-expr/common.sh's all_source_nodes
                           (an awk reader) returns for each list
"""
from __future__ import annotations

import importlib.util
import os
import random
import shutil
import subprocess
import sys
import tempfile

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "xblossom-sigmetrics27-ae_b200"))
import xbtrav  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))
if len(sys.argv) < 2:
    sys.exit("usage: make_format_golden.py <reference checkout>")
REF = sys.argv[1]

TRICKY = """# source list with the forms the experiment scripts accept
   # indented comment line
3
5 7   9
11 # a trailing comment

  13\t17
# 99 commented out
19
"""


def load_module(path: str, name: str):
    spec = importlib.util.spec_from_file_location(name, path)
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def awk_ids(path: str) -> list[int]:
    script = f'source "{REF}/scripts/4-expr/common.sh" && all_source_nodes "{path}"'
    out = subprocess.run(["bash", "-c", script], capture_output=True, text=True, check=True).stdout
    return [int(x) for x in out.split()]


def main() -> None:
    g = xbtrav.HostCSR.rmat(7, 4, seed=0x5EED)
    g.save_text(os.path.join(OUT, "formats_rmat7_rowOffsets.txt"), os.path.join(OUT, "formats_rmat7_colIndices.txt"))
    with tempfile.TemporaryDirectory() as tmp:
        row, col = os.path.join(tmp, "rmat7_rowOffsets.txt"), os.path.join(tmp, "rmat7_colIndices.txt")
        g.save_text(row, col)
        mm = load_module(f"{REF}/scripts/2-datasets/gunrock/csr_to_gunrock_mm.py", "ref_mm")
        mm.convert_to_mtx(row, col, os.path.join(OUT, "formats_rmat7.mtx"))
        lg = load_module(f"{REF}/scripts/2-datasets/ligra/csr_to_ligra_adj.py", "ref_ligra")
        lg.convert_to_ligra(row, col, os.path.join(OUT, "formats_rmat7.ligra"))
        sl = load_module(f"{REF}/scripts/2-datasets/src_nodes/generate_src_lists.py", "ref_src")
        random.seed(5)
        sl.analyze_graph(row, col, os.path.join(tmp, "rmat7"), 12)
        shutil.copy(os.path.join(tmp, "rmat7_src_nodes.txt"), os.path.join(OUT, "formats_rmat7_src_nodes.txt"))
    tricky = os.path.join(OUT, "formats_sources_tricky.txt")
    with open(tricky, "w") as f:
        f.write(TRICKY)
    for name in ("formats_rmat7_src_nodes", "formats_sources_tricky"):
        ids = awk_ids(os.path.join(OUT, name + ".txt"))
        with open(os.path.join(OUT, name + ".ids"), "w") as f:
            f.write(" ".join(map(str, ids)) + "\n")
        print(name, ids)


if __name__ == "__main__":
    main()
