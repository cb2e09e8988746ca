"""Writes reference_kat.json: the reference's own known answers and edge inputs.

Every value below is transcribed from a test in tomet-lang/oneline (the file and
lines are recorded next to each entry). The reference is Rust and cannot be run
in this environment, so these known answers are what pin the oracle; the edge
inputs feed the differential tests (oracle vs the CUDA path).

Run:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os

NONE = 0xFFFFFFFF
KIND = {"Blank": 0, "Text": 1, "Heading": 2, "Element": 3, "List": 4, "Connect": 5, "OrderedList": 6, "Comment": 7}


KAT = {
    "scan_line_offsets": [
        {"src": "crates/oneline-simd/src/lib.rs:530-535", "text": "line1\nline2\r\nline3\n", "offsets": [0, 6, 13]},
        {"src": "crates/oneline-gpu/src/tests.rs:75-83",
         "text": "|=[ Header ]\n| Body text\n||:rule(x)\n|| Content.\n", "offsets": [0, 13, 25, 36]},
    ],
    "parse_line": [
        # crates/oneline-simd/src/lib.rs:537-563 (depth, kind) of single lines
        {"src": "crates/oneline-simd/src/lib.rs:539-541", "line": "| @card(title:\"test\")\n", "depth": 1, "kind": KIND["Element"]},
        {"src": "crates/oneline-simd/src/lib.rs:543-545", "line": "||:rule(allow:list(card))\n", "depth": 2, "kind": KIND["Connect"]},
        {"src": "crates/oneline-simd/src/lib.rs:547-549", "line": "|||- List item\n", "depth": 3, "kind": KIND["List"]},
        {"src": "crates/oneline-simd/src/lib.rs:551-553", "line": "|-. Ordered\n", "depth": 1, "kind": KIND["OrderedList"]},
        {"src": "crates/oneline-simd/src/lib.rs:554", "line": "-.x\n", "kind": KIND["Text"]},
        {"src": "crates/oneline-simd/src/lib.rs:555", "line": "|| // c\n", "kind": KIND["Comment"]},
        {"src": "crates/oneline-simd/src/lib.rs:556", "line": "/x\n", "kind": KIND["Text"]},
        {"src": "crates/oneline-simd/src/lib.rs:558-560", "line": "|=[ Header ]\n", "depth": 1, "kind": KIND["Heading"]},
    ],
    "parse_document": [
        {"src": "crates/oneline-simd/src/lib.rs:565-576",
         "text": "|=[ Header ]\n| Is this syntax necessary?\n||:rule(x)\n|| Body text.\n",
         "depth_kind": [[1, KIND["Heading"]], [1, KIND["Text"]], [2, KIND["Connect"]], [2, KIND["Text"]]]},
        {"src": "crates/oneline-gpu/src/tests.rs:29-51",
         "text": "|=[ Header ]\n| Body text\n||:rule(x)\n|| Content.\n",
         "depth_kind": [[1, KIND["Heading"]], [1, KIND["Text"]], [2, KIND["Connect"]], [2, KIND["Text"]]]},
    ],
    "tree": [
        {"src": "crates/oneline-core/src/links.rs:90-111",
         # (depth, kind) per line: d 1 2 3 2 (blank) 1 0
         "nodes": [[1, 1], [2, 1], [3, 1], [2, 1], [0, 0], [1, 1], [0, 1]],
         "parent": [NONE, 0, 1, 0, NONE, NONE, NONE],
         "subtree_end": [5, 3, 3, 5, 5, 6, 7]},
    ],
    "find_all": [
        {"src": "crates/oneline-simd/src/search.rs:131", "text": "aaaa", "pattern": "aa", "offsets": [0, 1, 2]},
        {"src": "crates/oneline-simd/src/search.rs:132", "text": "abcabc", "pattern": "abc", "offsets": [0, 3]},
        {"src": "crates/oneline-simd/src/search.rs:133", "text": "abc", "pattern": "abcd", "offsets": []},
        {"src": "crates/oneline-simd/src/search.rs:134", "text": "", "pattern": "a", "offsets": []},
        {"src": "crates/oneline-simd/src/search.rs:135", "text": "xabc", "pattern": "abc", "offsets": [1]},
        {"src": "crates/oneline-simd/src/search.rs:136", "text": "a\nb", "pattern": "a\nb", "offsets": [0]},
        {"src": "crates/oneline-simd/src/search.rs:126", "text": "aaaa", "pattern": "aa", "count": 3},
    ],
    "query_raw": [
        {"src": "crates/oneline-gpu/src/tests.rs:86-107",
         "text": "| @card(title:\"A\")\n|| Content\n| @card(title:\"B\")\n|| More\n|=[ Header ]\n",
         "kind_element": [0, 2], "depth_2": [1, 3]},
    ],
    "tree_depth_limit": [
        {"src": "crates/oneline-gpu/src/tests.rs:571-591",
         "ok": ["|" * 31 + " x\n", "| a\n" + "|" * 40 + "\n| b\n"],
         "too_deep": ["| a\n" + "|" * 32 + " x\n| b\n"]},
    ],
}

EDGE_INPUTS = {
    # crates/oneline-simd/src/lib.rs:578-604
    "simd_edge_cases": ["", "\n", "\n\n\n", "x", "x\n", "x\ny", "\r\n", "a\r\nb\r\n", "|\n", "||||\n|||| \n",
                        "   \n\t\n", "| 日本語\n|| ｗｉｄｅ\n", "```\n- not a list\n```\n", "no trailing newline"],
    # crates/oneline-gpu/src/tests.rs:114-156
    "gpu_grammar_cases": ["x", "x\n", "\n", "\r\n", "a\r\nb", "||||\n|||| \n", "```\n- x\n```\n", "| 日本語\n",
                          "-\tx\n", "- x\n", "-x\n", "-\n", "- \n", ":rule(a)\n|| :{y:2}\n", "=\n=[ t ]\n", "@\n",
                          "> a\n* b\n1. c\n", "|-\tx\n|:y\n", "// c\n", "//\n", "/x\n", "/\n", "|| // c\n",
                          "http://x\n", "/// doc\n", "| | x\n", "|  | x\n", "|\t|x\n", "| x | y\n", "| |\n",
                          "|| |\n", " | x\n", "|| \t | \n", "-. x\n", "-.\tx\n", "-.x\n", "-.\n", "-. \n", "-..\n",
                          "- -. x\n"],
    # crates/oneline-gpu/src/tests.rs:56-71
    "gpu_scan_cases": ["hello", "hello\n", "line1\nline2\nline3\n", "line1\r\nline2\r\nline3\r\n", "\n\n\n",
                       "|=[ Header ]\n| Paragraph\n|| Content\n"],
    # crates/oneline-gpu/src/tests.rs:334-350: (text, pattern)
    "search_cases": [["aaaaaaaa", "aa"], ["abc", "abc"], ["xxabc", "abc"], ["ab", "abc"], ["a\nb\na\nb", "a\nb"],
                     ["xa", "a\u0000"], ["xa\u0000", "a\u0000"]],
    # crates/oneline-gpu/src/tests.rs:432-448: a window hit implying a start before the text
    "search_before_text": [["bcdq" + "\u0000" * 5000 + "xyz", "\u0000bcdq"]],
    # crates/oneline-gpu/src/tests.rs:805-861 (patterns shorter than 4 bytes dropped as there)
    "many_nested": {"text": "abcdefabcdefabcd\u0000\u0000\u0000\u0000abcdxabcdef|||||- - -\nabcdabcd",
                    "patterns": ["abcd", "abcdef", "bcde", "abcdef", "cdefabcd", "abcdabcd", "\u0000\u0000\u0000\u0000",
                                 "||||", "- - -", "abcdx", "xxxx-not-there", "abcdabcd"]},
    "many_whole_text": {"text": "abcdefgh", "patterns": ["abcdefgh", "abcd", "efgh"]},
    "many_longer_than_text": {"text": "abcdefgh", "patterns": ["abcdefghi", "zzzz"]},
}


def main() -> None:
    out = {"about": "Known answers and edge inputs transcribed from tomet-lang/oneline tests; "
                    "strings are the UTF-8 encoding of the bytes (the reference inputs are Rust &str or ASCII byte strings).",
           "kat": KAT, "edge_inputs": EDGE_INPUTS}
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "reference_kat.json")
    with open(path, "w", encoding="utf-8") as f:
        json.dump(out, f, ensure_ascii=False, indent=1)
    print(path)


if __name__ == "__main__":
    main()
