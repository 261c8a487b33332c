"""Generates the golden fixtures in this directory.

Inputs come from libchsga's seeded generator and hierarchy builder; expected
outputs come from the reference's OWN alignment code (src/align.hpp,
src/traceback.hpp, src/ParSGAoverrides/csr_align.hpp) compiled into
oracle/_ref by oracle/Makefile, so the fixtures pin both the CPU oracle and
the GPU path to the reference on machines where the reference tree is absent.

    python tests/golden/make_golden.py      # needs oracle/_ref built

Fixtures:
  hand.*        the hand DAG A -> {C, T} -> G (single-char vertices), reads
                ACG ATG AG ANG; expected scores 0 0 1 1
  g1.*          cfg1-style graph on a 3 kbp backbone, string vertices of
                1..32 chars, 12 reads of 40..150 bp
  g1.expected.json   reference scores (align_combo), exact-DP scores
                (serial_align_CSR), checkpoint rows of read 0 with k=16
                (checkpointed traceback, cleanup off) as row index -> sha256
  g1.rows0.npz  every DP row of read 0 (align_read_combo's rows), int16,
                compressed
"""
import hashlib
import json
import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import chsga_b200 as cb  # noqa: E402
import oracle  # noqa: E402


def write_hand(prefix):
    """A(0) -> C(1), A(0) -> T(2), C -> G(3), T -> G(3): one char per vertex."""
    labels = b"ACTG"
    edges = {0: [1, 2], 1: [3], 2: [3], 3: []}

    def adj(path):
        offs, tgts = [], []
        for u in range(4):
            offs.append(len(tgts))
            tgts.extend(edges[u])
        with open(path, "w") as f:
            f.write("AdjacencyGraph\n4\n%d\n" % len(tgts))
            f.write("".join("%d\n" % o for o in offs))
            f.write("".join("%d\n" % t for t in tgts))
            f.write("1.0\n" * len(tgts))

    adj(prefix + ".char.adj")
    adj(prefix + ".string.adj")
    with open(prefix + ".char.labels", "wb") as f:
        f.write(labels)
    with open(prefix + ".string.label_offsets", "w") as f:
        f.write("0 1 2 3 4\n")
    g = cb.HostGraph.read_files(prefix + ".char.adj", prefix + ".string.adj",
                                _pch_for(prefix), prefix + ".char.labels",
                                prefix + ".string.label_offsets")
    return g


def _pch_for(prefix):
    """Builds the hierarchy of prefix.string.adj with the build_pch tool."""
    import subprocess
    out = prefix + ".string.out"
    subprocess.run([os.path.join(ROOT, "chsga_b200", "bin", "build_pch"), "-i",
                    prefix + ".string.adj", "-o", out, "-v", prefix + ".string.label_offsets"],
                   check=True, stdout=subprocess.DEVNULL)
    return out


def main():
    assert oracle.ref_available(), "build oracle/_ref first (make -C oracle ref)"
    # hand DAG
    hp = os.path.join(HERE, "hand")
    write_hand(hp)
    hand_files = cb.files_for(hp)
    hand_reads = [b"ACG", b"ATG", b"AG", b"ANG"]
    ref = oracle.RefHarness(hand_files)
    hand = {"reads": [r.decode() for r in hand_reads],
            "scores": ref.scores(hand_reads).tolist(),
            "exact": ref.exact_scores(hand_reads).tolist()}
    assert hand["scores"] == [0, 0, 1, 1], hand
    with open(os.path.join(HERE, "hand.expected.json"), "w") as f:
        json.dump(hand, f, indent=1)

    # cfg1-style graph
    cfg = dict(cb.GRAPH_CONFIGS["cfg1"])
    cfg.update(backbone_len=3000, seed=101, bubble_gap_mean=20.0, p_snp=0.6, p_indel=0.3,
               p_alt=0.1, alt_min=5, alt_max=60)
    g = cb.HostGraph.generate(**cfg).build_pch()
    gp = os.path.join(HERE, "g1")
    files = g.write_files(gp)
    reads = g.gen_reads(12, 102, 40, 150, sub_rate=0.03, indel_rate=0.02, n_rate=0.01).to_list()
    with open(gp + ".reads.fa", "w") as f:
        for i, r in enumerate(reads):
            f.write(">r%d\n%s\n" % (i, r.decode()))
    ref = oracle.RefHarness(files)
    scores = ref.scores(reads).tolist()
    exact = ref.exact_scores(reads).tolist()
    num_chars = len(open(files[3], "rb").read().replace(b"\n", b""))
    rows0 = ref.rows(reads[0], num_chars)
    assert rows0.max() < 2 ** 15
    np.savez_compressed(gp + ".rows0.npz", rows=rows0.astype(np.int16))
    ck = oracle.RefHarness(files, checkpointed=True)
    with tempfile.TemporaryDirectory() as d:
        ops = ck.traceback(reads[0], k=16, ckpt_dir=d, cleanup=False)
        rows = {}
        for name in sorted(os.listdir(d)):
            i = int(name[4:-4])
            rows[i] = hashlib.sha256(open(os.path.join(d, name), "rb").read()).hexdigest()
    labels = open(files[3], "rb").read().replace(b"\n", b"")
    ps, last = oracle.rescore(ops, reads[0], labels)
    exp = {"reads": [r.decode() for r in reads], "scores": scores, "exact": exact,
           "num_chars": num_chars, "ckpt_k": 16,
           "ckpt_rows_sha256": {str(k): v for k, v in sorted(rows.items())},
           "ckpt_path_score": ps, "ckpt_last_row": last}
    assert ps == scores[0] and last == len(reads[0]) - 1
    with open(gp + ".expected.json", "w") as f:
        json.dump(exp, f, indent=1)
    print("golden fixtures written:", scores)


if __name__ == "__main__":
    main()
