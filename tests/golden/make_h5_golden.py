"""Writes tests/golden/h5_legacy_messages.json from the reference's HDF5 fixtures
(tests/io/fixtures/legacy*.h5 of the reference, written by the HDF5 library through ESIO): for
every dataset the raw bodies of its dataspace, datatype and fill-value messages, the flags of
each message type, its comment and attributes, and its data bytes, read with the independent
walker tests/h5walk.py.  The checkpoint tests compare the library's own writer and reader with
these without needing the reference checkout.

    python tests/golden/make_h5_golden.py [fixtures directory]
"""
import json
import os
import sys

sys.path.insert(0, os.path.join(os.path.dirname(__file__), "..", ".."))
from tests.h5walk import H5Walk  # noqa: E402

SRC = sys.argv[1] if len(sys.argv) > 1 else "/root/reference/SOURCE_PASSOPB/tests/io/fixtures"
OUT = os.path.join(os.path.dirname(__file__), "h5_legacy_messages.json")


def attr_body(body):
    return body.hex()


def main():
    out = {}
    for fn in sorted(os.listdir(SRC)):
        if not fn.endswith(".h5"):
            continue
        w = H5Walk(os.path.join(SRC, fn))
        sets = {}
        for name in sorted(w.links):
            m = w.dataset(name)
            sets[name] = {
                "dataspace": m[0x01][1].hex(),
                "datatype": m[0x03][1].hex(),
                "fill": m[0x05][1].hex(),
                "flags": {hex(t): fl for t, (fl, _) in m.items()},
                "comment": m[0x0D][1].split(b"\0")[0].decode() if 0x0D in m else "",
                "attributes": [b.hex() for t, fl, b in w.messages(w.links[name]) if t == 0x0C],
                "data": w.data(name).hex(),
            }
        out[fn] = {
            "leaf_k": w.leaf_k, "node_k": w.node_k,
            "root_attributes": [b.hex() for t, fl, b in w.root_msgs if t == 0x0C],
            "btree_keys": w.btree_keys,
            "datasets": sets,
        }
    with open(OUT, "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)
    print(OUT, sum(len(v["datasets"]) for v in out.values()), "datasets")


if __name__ == "__main__":
    main()
