"""Reference arm of bench.py: placeholder until the reference-run driver lands."""
import json


def run(a):
    print(json.dumps({"impl": "reference", "unavailable": "reference arm not wired yet"}))
