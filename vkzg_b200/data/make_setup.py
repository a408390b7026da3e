"""Extracts the Ethereum mainnet KZG ceremony's 4096 compressed G1 monomial points
([tau^i]G1, 48 bytes each) from jtraglia/vkzg's src/setup_data.cpp into
trusted_setup_g1_monomial.bin, checking the sha256 that src/setup_data.h:13 records.

This is protocol data (the public ceremony output), not code: the bytes must be the
same in every EIP-7594 implementation.

    python vkzg_b200/data/make_setup.py <reference checkout>/src/setup_data.cpp

(or with $VKZG_REFERENCE_DIR set and no argument).
"""
import hashlib
import os
import re
import sys

SHA256 = "08797579f6cfd5788eddc1a215d64dcfabd04acbcaf2953fb2c1afb830f43315"


def main(src):
    text = open(src).read()
    body = text[text.index("{", text.index("kEmbeddedSetupG1Monomial")) + 1:text.rindex("}", 0, text.rindex("namespace"))]
    data = bytes(int(h, 16) for h in re.findall(r"0x([0-9a-fA-F]{2})", body))
    assert len(data) == 4096 * 48, len(data)
    assert hashlib.sha256(data).hexdigest() == SHA256
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "trusted_setup_g1_monomial.bin")
    open(out, "wb").write(data)
    print("wrote", out)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("VKZG_REFERENCE_DIR"):
        main(os.path.join(os.environ["VKZG_REFERENCE_DIR"], "src", "setup_data.cpp"))
    else:
        sys.exit("usage: make_setup.py <reference checkout>/src/setup_data.cpp (or set VKZG_REFERENCE_DIR)")
