"""Generates tests/golden/ref_kernels_golden.json: outputs of the REFERENCE's own CUDA kernels
(oracle/_ref/libbcref.so, built from crates/boojum-cuda/native by oracle/build_ref.py) on
seeded synthetic inputs.  Run on a machine with a GPU:

    python tests/golden/make_golden.py [out.json]

Each case stores its parameters, the seed of its input (zksync-crypto-gpu_b200/synthetic.py
ChaCha20 stream), the SHA-256 of the canonical little-endian output and its first elements.
The Poseidon2 cases also record the SHA-256 of the round constants they were made with.
"""
import hashlib
import importlib
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))
P = 0xFFFFFFFF00000001


def digest(a):
    a = np.asarray(a, dtype=np.uint64)
    a = np.where(a >= np.uint64(P), a - np.uint64(P), a)
    return hashlib.sha256(a.astype("<u8").tobytes()).hexdigest(), [int(v) for v in a[:4]]


def ntt_cases():
    out = []
    for log_n in (1, 2, 3, 5, 8, 11, 12, 13, 15, 16, 17, 20):
        for bitrev in (False, True):
            for inverse in (False, True):
                for log_ext, coset in ((0, 0), (3, 3), (1, 1)):
                    cols = 3 if log_n <= 13 else 1
                    out.append(dict(kind="ntt", log_n=log_n, cols=cols, bitrev_inputs=bitrev, inverse=inverse,
                                    log_ext=log_ext, coset=coset, seed="ntt-%d-%d-%d-%d-%d" % (log_n, bitrev, inverse, log_ext, coset)))
    return out


def main(path):
    import torch
    import refkern
    syn = importlib.import_module("zksync-crypto-gpu_b200.synthetic")
    consts = importlib.import_module("zksync-crypto-gpu_b200.p2_constants")
    rc = consts.env_round_constants() or consts.grain_lfsr_round_constants()
    rc_hash = hashlib.sha256(np.array(rc, dtype="<u8").tobytes()).hexdigest()
    refkern.call("ref_context_create", 12, 12)
    s = torch.cuda.current_stream().cuda_stream

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint64).view(np.int64).copy()).cuda()

    def host(t):
        torch.cuda.synchronize()
        return t.cpu().numpy().view(np.uint64)

    cases = []
    for c in ntt_cases():
        n = 1 << c["log_n"]
        x = syn.random_field_elements(c["seed"], c["cols"] * n)
        d_in, d_out = dev(x), torch.zeros(c["cols"] * n, dtype=torch.int64, device="cuda")
        refkern.call("ref_batch_ntt", d_in.data_ptr(), d_out.data_ptr(), c["log_n"], c["cols"], n, n,
                     c["bitrev_inputs"], c["inverse"], c["log_ext"], c["coset"], s)
        c["sha256"], c["head"] = digest(host(d_out))
        cases.append(c)
    for log_n in (4, 10, 11):
        n = 1 << log_n
        x = syn.random_field_elements("bitrev-%d" % log_n, 2 * n)
        d_in, d_out = dev(x), torch.zeros(2 * n, dtype=torch.int64, device="cuda")
        refkern.call("ref_bit_reverse", d_in.data_ptr(), n, d_out.data_ptr(), n, log_n, 2, s)
        h, head = digest(host(d_out))
        cases.append(dict(kind="bitrev", log_n=log_n, cols=2, seed="bitrev-%d" % log_n, sha256=h, head=head))
    for log_n, cols, log_rows in ((4, 9, 1), (8, 9, 1), (6, 8, 0), (6, 3, 2)):
        count = 1 << log_n
        x = syn.random_field_elements("leaves-%d-%d-%d" % (log_n, cols, log_rows), cols * count << log_rows)
        d_in, d_out = dev(x), torch.zeros(4 * count, dtype=torch.int64, device="cuda")
        refkern.call("ref_p2_leaves", d_in.data_ptr(), x.size, d_out.data_ptr(), 4 * count, log_rows, False, False, s)
        h, head = digest(host(d_out))
        cases.append(dict(kind="leaves", log_n=log_n, cols=cols, log_rows=log_rows, rc_sha256=rc_hash,
                          seed="leaves-%d-%d-%d" % (log_n, cols, log_rows), sha256=h, head=head))
    for log_n in (3, 9):
        count = 1 << log_n
        x = syn.random_field_elements("nodes-%d" % log_n, 8 * count)
        d_in, d_out = dev(x), torch.zeros(4 * count, dtype=torch.int64, device="cuda")
        refkern.call("ref_p2_nodes", d_in.data_ptr(), 8 * count, d_out.data_ptr(), 4 * count, s)
        h, head = digest(host(d_out))
        cases.append(dict(kind="nodes", log_n=log_n, rc_sha256=rc_hash, seed="nodes-%d" % log_n, sha256=h, head=head))
    for log_n, cols, layers in ((10, 9, 11), (10, 5, 7)):
        n = 1 << log_n
        x = syn.random_field_elements("tree-%d-%d" % (log_n, cols), cols * n)
        d_in, d_out = dev(x), torch.zeros(8 * n, dtype=torch.int64, device="cuda")
        refkern.call("ref_p2_build_merkle_tree", d_in.data_ptr(), x.size, d_out.data_ptr(), 8 * n, 0, layers, s)
        h, head = digest(host(d_out))
        cases.append(dict(kind="tree", log_n=log_n, cols=cols, layers=layers, rc_sha256=rc_hash,
                          seed="tree-%d-%d" % (log_n, cols), sha256=h, head=head))
    with open(path, "w") as f:
        json.dump({"generator": "reference kernels (crates/boojum-cuda/native) on sm_100a via oracle/ref_harness.cu",
                   "cases": cases}, f, indent=1)
    print("wrote", path, len(cases), "cases")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(os.path.abspath(__file__)),
                                                            "ref_kernels_golden.json"))
