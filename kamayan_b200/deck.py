"""Parthenon-style input decks for kamayan_b200.

Mirrors the reference's input-file handling (``<block>`` headers with
``key = value`` lines and ``block/key=value`` command-line overrides,
parthenon ParameterInput as used by kamayan's RuntimeParameters,
src/kamayan/runtime_parameters.hpp:177-234).  The C library parses the same
text; this module only assembles and edits decks on the host.
"""
from __future__ import annotations

from collections import OrderedDict


class Deck:
    """Ordered {block: {key: value}} with Parthenon text round-tripping."""

    def __init__(self, blocks: dict | None = None):
        self.blocks: OrderedDict[str, OrderedDict[str, str]] = OrderedDict()
        for b, kv in (blocks or {}).items():
            for k, v in kv.items():
                self.set(b, k, v)

    @classmethod
    def parse(cls, text: str) -> "Deck":
        d = cls()
        block = ""
        for raw in text.splitlines():
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            if line.startswith("<") and line.endswith(">"):
                block = line[1:-1].strip()
                continue
            if "=" not in line:
                continue
            k, v = (s.strip() for s in line.split("=", 1))
            if "/" in k:
                b, k = k.rsplit("/", 1)
                d.set(b, k, v)
            else:
                d.set(block, k, v)
        return d

    def set(self, block: str, key: str, value) -> "Deck":
        self.blocks.setdefault(block, OrderedDict())[key] = _fmt(value)
        return self

    def get(self, block: str, key: str, default=None):
        return self.blocks.get(block, {}).get(key, default)

    def override(self, *args: str) -> "Deck":
        """Apply ``block/key=value`` overrides (the reference's command-line form)."""
        for a in args:
            k, v = a.split("=", 1)
            b, key = k.strip().rsplit("/", 1)
            self.set(b, key, v.strip())
        return self

    def __setitem__(self, block: str, values) -> None:
        """``deck["hydro"] = {"reconstruction": "wenoz"}``: set several keys of a
        block at once, the way the reference's KamayanParams does
        (python/kamayan/code_units/parameters.py, ``__setitem__``)."""
        for k, v in values.items():
            self.set(block, k, v)

    def __getitem__(self, block: str) -> dict:
        return dict(self.blocks.get(block, {}))

    def write(self, path, problem_id: str | None = None) -> None:
        """Write the deck as an input file.  With ``problem_id`` the file opens
        with a ``<parthenon/job>`` block naming it, as the reference's
        KamayanManager.write_input does (python/kamayan/kamayan_manager.py:123-156)."""
        d = self.copy()
        if problem_id is not None:
            rest = OrderedDict((b, kv) for b, kv in d.blocks.items() if b != "parthenon/job")
            job = OrderedDict(d.blocks.get("parthenon/job", {}))
            job["problem_id"] = str(problem_id)
            d.blocks = OrderedDict([("parthenon/job", job)] + list(rest.items()))
        with open(path, "w") as f:
            f.write(d.text())

    def copy(self) -> "Deck":
        return Deck({b: dict(kv) for b, kv in self.blocks.items()})

    def text(self) -> str:
        out = []
        for b, kv in self.blocks.items():
            out.append(f"<{b}>")
            out.extend(f"{k} = {v}" for k, v in kv.items())
            out.append("")
        return "\n".join(out)

    __str__ = text


def _fmt(v) -> str:
    if isinstance(v, bool):
        return "true" if v else "false"
    if isinstance(v, float):
        return repr(v)
    return str(v)


def deck_text(blocks: dict) -> str:
    return Deck(blocks).text()
