"""Extracts a few Merkle openings (leaf elements, sibling path) and the caps they open against
from the reference's proof fixtures into this directory:
  * crates/shivini/test_data/compression/scheduler_recursive_proof.json -> scheduler_proof_openings.json
  * crates/shivini/test_data/base/1.cpu.proof (bincode) -> base_proof_openings.json: the witness
    cap, the distinct last path elements of the 100 queries (the nodes one level below the cap)
    and two openings.
Run once where the reference is mounted:

    python tests/golden/extract_proof_openings.py /root/reference
"""
import json
import os
import sys

ref = sys.argv[1] if len(sys.argv) > 1 else "/root/reference"
src = os.path.join(ref, "crates/shivini/test_data/compression/scheduler_recursive_proof.json")
d = json.load(open(src))["SchedulerCircuit"]
caps = {"witness": d["witness_oracle_cap"], "stage_2": d["stage_2_oracle_cap"], "quotient": d["quotient_oracle_cap"]}
queries = []
for rep in d["queries_per_fri_repetition"][:2]:
    for name in ("witness", "stage_2", "quotient"):
        q = rep[name + "_query"]
        queries.append({"oracle": name, "leaf_elements": q["leaf_elements"], "proof": q["proof"]})
out = {"source": "crates/shivini/test_data/compression/scheduler_recursive_proof.json",
       "proof_config": d["proof_config"], "caps": caps, "queries": queries}
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "scheduler_proof_openings.json"), "w") as f:
    json.dump(out, f)
print(len(queries), "openings")

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import round_constant_candidates as rcc  # noqa: E402

caps, bq = rcc.parse_bincode_proof(os.path.join(ref, "crates/shivini/test_data/base/1.cpu.proof"))
sib = sorted({tuple(q["witness"]["proof"][-1]) for q in bq})
with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "base_proof_openings.json"), "w") as f:
    json.dump({"source": "crates/shivini/test_data/base/1.cpu.proof (bincode Proof, tree hasher GLHasher)",
               "witness_cap": caps["witness"], "last_level_siblings": [list(s) for s in sib],
               "witness_openings": [q["witness"] for q in bq[:2]]}, f)
print(len(sib), "last-level siblings")
