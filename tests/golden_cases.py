import json
import os

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def cases():
    return sorted(d for d in os.listdir(GOLDEN) if os.path.exists(os.path.join(GOLDEN, d, "case.json")))


def load(name):
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, "case.json")) as f:
        return d, json.load(f)
