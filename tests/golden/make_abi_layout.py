"""Writes tests/golden/abi_layout_ref.json: sizeof / offsetof of every
struct of fp_cuda_backend.h (field list from this repository's header)
compiled against the reference's own headers (include/fp_cuda_backend.h,
include/fp_shared_core.h, include/params.h) at np = npe = 128, 256, 512.

    python tests/golden/make_abi_layout.py [<reference checkout>]

(default: $CROMA_REFERENCE_ROOT, else /root/reference)."""
import json
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))

from abi_layout import measure_all, struct_fields  # noqa: E402

if __name__ == "__main__":
    ref = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("CROMA_REFERENCE_ROOT", "/root/reference")
    res = measure_all(os.path.join(ref, "include"), struct_fields())
    json.dump(res, open(os.path.join(HERE, "abi_layout_ref.json"), "w"), indent=0, sort_keys=True)
    print("abi_layout_ref.json written:", {k: len(v) for k, v in res.items()}, "entries")
