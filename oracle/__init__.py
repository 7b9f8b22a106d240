"""CPU checkers (test infrastructure only): the FP64 C oracle and the reference
binaries built from the reference sources.  Never imported by the product."""
