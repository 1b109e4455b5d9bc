"""Index format conversion between the reference's two on-disk layouts:

    python -m mvr.convert plaid2igp <plaid index dir> <igp index dir>
    python -m mvr.convert igp2plaid <igp index dir> <plaid index dir> <n_bit>

An IGP index directory (item_n_vec_l.npy, centroid_l.npy, vq_code_l.npy,
weight_l.npy, residual_code_l.npy, ivf.index) is what the IGPGPUBasic /
IGPGPUPP executables and mvr_index_load read; a PLAID directory is what the
reference's ColBERT baseline writes.  The conversion keeps centroids, codes,
bucket weights and IVF lists and re-lays the residual bits (formats.py);
PLAID stores centroids and weights in fp16, so igp2plaid rounds them.
"""
import sys

from . import formats


def plaid_to_igp(src, dst):
    ix = formats.read_plaid_index(src)
    formats.write_index_dir(dst, ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["weight"],
                            ix["residual"], ix["ivf_off"], ix["ivf_size"], ix["ivf_ids"])
    return ix


def igp_to_plaid(src, dst, n_bit):
    ix = formats.read_index_dir(src)
    formats.write_plaid_index(dst, ix["item_n_vec"], ix["centroid"], ix["vq_code"], ix["weight"],
                              ix["residual"], ix["ivf_off"], ix["ivf_size"], ix["ivf_ids"],
                              int(n_bit))
    return ix


def main(argv):
    if len(argv) >= 3 and argv[0] == "plaid2igp":
        ix = plaid_to_igp(argv[1], argv[2])
    elif len(argv) >= 4 and argv[0] == "igp2plaid":
        ix = igp_to_plaid(argv[1], argv[2], argv[3])
    else:
        print(__doc__)
        return 2
    print(f"{len(ix['item_n_vec'])} docs, {len(ix['vq_code'])} vectors, "
          f"{len(ix['ivf_size'])} centroids -> {argv[2]}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))
