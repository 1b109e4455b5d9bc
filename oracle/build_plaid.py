"""Compiles the reference's own PLAID CPU search extensions from their
sources where they lie (baseline/ColBERT/colbert/search/filter_pids.cpp,
search/decompress_residuals.cpp, modeling/segmented_maxsim.cpp) into
oracle/_ref/plaid/<name>/<name>.so with torch's extension builder -- the
recipe the reference's own loaders use (index_storage.py:37-61,
colbert.py:39-50), pointed at a build folder inside this repository.  Test
and baseline infrastructure only: plaid_cpu.py loads the built modules.

    python oracle/build_plaid.py [reference root, default MVR_REFERENCE_ROOT]
"""
import os
import sys

from refroot import REF_ROOT

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref", "plaid")
SOURCES = {
    "filter_pids_cpp": "baseline/ColBERT/colbert/search/filter_pids.cpp",
    "decompress_residuals_cpp": "baseline/ColBERT/colbert/search/decompress_residuals.cpp",
    "segmented_maxsim_cpp": "baseline/ColBERT/colbert/modeling/segmented_maxsim.cpp",
}


def main(ref_root=REF_ROOT):
    from torch.utils.cpp_extension import load
    for name, rel in SOURCES.items():
        src = os.path.join(ref_root, rel)
        if not os.path.exists(src):
            print(f"{src} absent: {name} not built")
            continue
        bdir = os.path.join(OUT, name)
        os.makedirs(bdir, exist_ok=True)
        load(name=name, sources=[src], extra_cflags=["-O3"], build_directory=bdir,
             verbose=False)
        print("built", os.path.join(bdir, name + ".so"))


if __name__ == "__main__":
    main(*sys.argv[1:])
