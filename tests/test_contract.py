"""Contract-v2 output (e-hgp_b200/contract.py) of the direct hierarchy.

* The critical catalogue equals, record for record and id for id, the one the
  reference's own contract serializer writes for the exhaustive oracle
  (reference/morsehgp3d_oracle/serialization.py; golden definition fixtures).
* The whole document validates against the contract's JSON schema when the
  reference tree (which holds the schema) is present.
* On the GPU, the document built from the device arrays is identical, byte for
  byte, to the one built from the restatement oracle's journal."""
import glob
import json
import os

import numpy as np
import pytest

import contract
from geomcheck import hier_dict_from_text
from oracle import pyoracle

DEFINITION = sorted(glob.glob(os.path.join(os.path.dirname(__file__), "golden", "definition_*.json")))
_REF = pyoracle.reference_root() or ""  # the reference checkout holds the schema
SCHEMA = os.path.join(_REF, "morsehgp3d", "schemas", "morsehgp3d-contract-v2.schema.json")
SCHEMA_ALT = os.path.join(_REF, "schemas", "morsehgp3d-contract-v2.schema.json")


def canonical_order(pts):
    order = np.lexsort((pts[:, 2], pts[:, 1], pts[:, 0]))
    return pts[order], order


def oracle_contract(pts, K):
    canon, order = canonical_order(pts)
    keff = min(K, len(pts))
    h = hier_dict_from_text(pyoracle.hierarchy(pts, K), len(pts), keff)
    return contract.build_contract(canon, order, K, h)


@pytest.mark.parametrize("path", DEFINITION, ids=[os.path.basename(p)[11:-5] for p in DEFINITION])
def test_catalog_matches_reference_serializer(path):
    d = json.load(open(path))
    doc = oracle_contract(np.array(d["points"]), d["K"])
    assert doc["critical_catalog"] == d["catalog"]


@pytest.mark.skipif(not (os.path.exists(SCHEMA) or os.path.exists(SCHEMA_ALT)), reason="contract schema absent")
@pytest.mark.parametrize("path", DEFINITION[:3], ids=[os.path.basename(p)[11:-5] for p in DEFINITION[:3]])
def test_contract_validates_against_schema(path):
    jsonschema = pytest.importorskip("jsonschema")
    schema = json.load(open(SCHEMA if os.path.exists(SCHEMA) else SCHEMA_ALT))
    d = json.load(open(path))
    doc = json.loads(contract.dumps(oracle_contract(np.array(d["points"]), d["K"])))
    errors = list(jsonschema.Draft202012Validator(schema).iter_errors(doc))
    assert not errors, errors[0].message


@pytest.mark.gpu
@pytest.mark.parametrize("path", DEFINITION, ids=[os.path.basename(p)[11:-5] for p in DEFINITION])
def test_gpu_contract_equals_oracle_contract(ctx, path):
    d = json.load(open(path))
    pts = np.array(d["points"])
    snap = ctx.lbvh_build(pts)
    canon = pts[np.asarray(snap.source_index, np.int64)]
    res = ctx.hierarchy(d["K"])
    ours = contract.build_contract(canon, np.asarray(snap.source_index), d["K"], res)
    assert contract.dumps(ours) == contract.dumps(oracle_contract(pts, d["K"]))
