import json
import os

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _all():
    return sorted(d for d in os.listdir(GOLDEN) if os.path.exists(os.path.join(GOLDEN, d, "case.json")))


def _is_d2(name):
    with open(os.path.join(GOLDEN, name, "case.json")) as f:
        return json.load(f)["command"].startswith("daligner2")


def cases():
    """Golden cases of the reference daligner (dalign/)."""
    return [d for d in _all() if not _is_d2(d)]


def d2_cases():
    """Golden cases of the reference daligner2 (dalign2/, modimizer seeds)."""
    return [d for d in _all() if _is_d2(d)]


def load(name):
    d = os.path.join(GOLDEN, name)
    with open(os.path.join(d, "case.json")) as f:
        return d, json.load(f)
