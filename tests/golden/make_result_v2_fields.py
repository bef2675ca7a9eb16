"""Writes result_v2_fields.json: the required fields, constants and enumerations of the
reference's result-v2 schema (spec/schemas/result-v2.schema.json), against which the
drop-in's restated artifact checks (foilbench_b200/results.py) are pinned.

    python tests/golden/make_result_v2_fields.py /root/reference
"""

import json
import sys
from pathlib import Path


def main(ref_root: str) -> None:
    schema = json.loads((Path(ref_root) / "spec" / "schemas" / "result-v2.schema.json").read_text())
    props = schema["properties"]
    out = {
        "required": schema["required"],
        "additional_properties": schema.get("additionalProperties", True),
        "consts": {k: v["const"] for k, v in props.items() if "const" in v},
        "enums": {k: v["enum"] for k, v in props.items() if "enum" in v},
    }
    dest = Path(__file__).resolve().parent / "result_v2_fields.json"
    dest.write_text(json.dumps(out, indent=1) + "\n")
    print(f"wrote {dest}")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference")
