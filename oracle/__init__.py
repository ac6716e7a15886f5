"""TEST INFRASTRUCTURE: CPU oracles (C restatement and the reference build)."""
