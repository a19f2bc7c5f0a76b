"""Embed the engine's CUDA sources as C++ raw-string constants (build step).

usage: python embed.py OUT.inc params.cuh common.cuh engine.cuh batched.cuh
"""
import sys


def raw(name: str, path: str) -> str:
    text = open(path, encoding="utf-8").read()
    delim = "MBSRC"
    assert ")" + delim + '"' not in text
    # string literals longer than ~64 KB are split into concatenated pieces
    pieces = [text[i:i + 30000] for i in range(0, len(text), 30000)] or [""]
    body = "\n".join(f'R"{delim}({p}){delim}"' for p in pieces)
    return f"static const char* const {name} =\n{body};\n"


def main() -> None:
    out, params, common, engine, batched = sys.argv[1:6]
    src = "// generated by embed.py -- do not edit\n"
    text = open(params, encoding="utf-8").read() + "\n" + open(common, encoding="utf-8").read()
    tmp = out + ".params.tmp"
    with open(tmp, "w", encoding="utf-8") as f:
        f.write(text)
    src += raw("mb_params_source", tmp) + raw("mb_engine_source", engine) + raw("mb_batched_source", batched)
    import os
    os.remove(tmp)
    with open(out, "w", encoding="utf-8") as f:
        f.write(src)


if __name__ == "__main__":
    main()
