"""The oracle against golden vectors made by the REFERENCE's own kernels (tests/golden/make_golden.py)
and against the Merkle openings recorded in the reference's proof fixture."""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import P, load_constants_module

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "ref_kernels_golden.json")
OPENINGS = os.path.join(HERE, "golden", "scheduler_proof_openings.json")
BASE_OPENINGS = os.path.join(HERE, "golden", "base_proof_openings.json")


def digest(a):
    a = np.asarray(a, dtype=np.uint64)
    a = np.where(a >= np.uint64(P), a - np.uint64(P), a)
    return hashlib.sha256(a.astype("<u8").tobytes()).hexdigest()


def golden_cases():
    if not os.path.exists(GOLDEN):
        return []
    with open(GOLDEN) as f:
        return json.load(f)["cases"]


def case_id(c):
    return "-".join(str(c.get(k)) for k in ("kind", "log_n", "cols", "bitrev_inputs", "inverse", "log_ext", "coset"))


@pytest.mark.skipif(not os.path.exists(GOLDEN), reason="golden vectors not generated yet")
@pytest.mark.parametrize("case", golden_cases(), ids=case_id)
def test_oracle_matches_reference_kernels(oracle, syn, round_constants, case):
    k = case["kind"]
    if "rc_sha256" in case:
        rc_hash = hashlib.sha256(np.array(round_constants, dtype="<u8").tobytes()).hexdigest()
        if rc_hash != case["rc_sha256"]:
            pytest.skip("golden Poseidon2 vectors were made with other round constants")
    if k == "ntt":
        n = 1 << case["log_n"]
        x = syn.random_field_elements(case["seed"], case["cols"] * n)
        y = oracle.batch_ntt(x, case["log_n"], case["cols"], n, n, case["bitrev_inputs"], case["inverse"],
                             case["log_ext"], case["coset"])
    elif k == "bitrev":
        n = 1 << case["log_n"]
        x = syn.random_field_elements(case["seed"], case["cols"] * n)
        y = oracle.bit_reverse(x, case["log_n"], case["cols"])
    elif k == "leaves":
        count = 1 << case["log_n"]
        x = syn.random_field_elements(case["seed"], case["cols"] * count << case["log_rows"])
        y = oracle.leaves(x, 4 * count, case["log_rows"])
    elif k == "nodes":
        count = 1 << case["log_n"]
        y = oracle.nodes(syn.random_field_elements(case["seed"], 8 * count))
    elif k == "tree":
        n = 1 << case["log_n"]
        x = syn.random_field_elements(case["seed"], case["cols"] * n)
        y = oracle.build_merkle_tree(x, 8 * n, 0, case["layers"])
    else:
        pytest.fail("unknown case kind %s" % k)
    assert [int(v) for v in y[:4]] == case["head"]
    assert digest(y) == case["sha256"]


@pytest.mark.skipif(not os.path.exists(OPENINGS), reason="proof openings not extracted")
def test_proof_fixture_openings(oracle):
    """Known-answer test from crates/shivini/test_data/compression/scheduler_recursive_proof.json:
    hashing a recorded leaf and climbing its recorded path must reach the recorded cap.  This pins
    the round constants, the sponge and the node order to boojum's; it needs boojum's real
    constants (GLC_P2_ROUND_CONSTANTS), which the reference tree does not contain."""
    consts = load_constants_module()
    rc = consts.env_round_constants()
    if rc is None:
        pytest.skip("parity unpinned: boojum's Poseidon2 round constants are not supplied "
                    "(set GLC_P2_ROUND_CONSTANTS to a file with the 360 values)")
    oracle.set_round_constants(rc)
    with open(OPENINGS) as f:
        data = json.load(f)
    for q in data["queries"]:
        cap = data["caps"][q["oracle"]]
        idx = oracle.find_opening(q["leaf_elements"], q["proof"], cap)
        assert idx >= 0, "opening of %s does not reach the cap" % q["oracle"]


@pytest.mark.skipif(not os.path.exists(BASE_OPENINGS), reason="proof openings not extracted")
def test_base_proof_fixture_cap(oracle):
    """Known-answer test from crates/shivini/test_data/base/1.cpu.proof (GLHasher): the nodes one
    level below the 16-entry witness cap, hashed pairwise, reproduce the cap (one node permutation
    per entry), and the recorded openings climb to it.  Needs boojum's real round constants;
    tests/golden/round_constant_candidates.json records the generated candidates that fail it."""
    import itertools
    consts = load_constants_module()
    rc = consts.env_round_constants()
    if rc is None:
        pytest.skip("parity unpinned: boojum's Poseidon2 round constants are not supplied "
                    "(set GLC_P2_ROUND_CONSTANTS to a file with the 360 values)")
    oracle.set_round_constants(rc)
    with open(BASE_OPENINGS) as f:
        data = json.load(f)
    cap = {tuple(c) for c in data["witness_cap"]}
    found = set()
    for a, b in itertools.permutations(data["last_level_siblings"], 2):
        out = oracle.permutation(np.array(list(a) + list(b) + [0] * 4, dtype=np.uint64))
        d = tuple(int(x) % P for x in out[:4])
        if d in cap:
            found.add(d)
    assert len(found) >= 12, "only %d of 16 cap entries reproduced" % len(found)
    for q in data["witness_openings"]:
        assert oracle.find_opening(q["leaf_elements"], q["proof"], data["witness_cap"]) >= 0


def test_candidate_record_is_negative():
    """The committed record of generated round-constant candidates: every candidate was checked
    against the base proof's cap and none reproduced it (parity against boojum stays unpinned)."""
    path = os.path.join(HERE, "golden", "round_constant_candidates.json")
    with open(path) as f:
        rec = json.load(f)
    assert len(rec["results"]) >= 40
    assert all(r["cap_pairs_reproduced"] == 0 and r["openings_verified"] == 0 for r in rec["results"])
