"""Writes tests/golden/wire_schema.json: the Params field paths and enum option strings the
reference's web client sends (web/src/params/schema.ts, the `path:` and `value: "..."` entries),
read as text from a MillDynamics3 checkout. Usage: python make_wire_schema.py <reference root>."""
import json
import os
import re
import sys

root = sys.argv[1]
text = open(os.path.join(root, "web", "src", "params", "schema.ts")).read()
fields = []
for m in re.finditer(r'path:\s*"([a-z_]+\.[a-z_0-9]+)"', text):
    nxt = text.find("path:", m.end())
    body = text[m.end():nxt if nxt >= 0 else len(text)]
    fields.append({"path": m.group(1), "options": re.findall(r'\{\s*value:\s*"([a-z_]+)"', body)})
out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "wire_schema.json")
with open(out, "w") as f:
    json.dump({"source": "web/src/params/schema.ts", "fields": fields}, f, indent=1)
print(out, len(fields))
