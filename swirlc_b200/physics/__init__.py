"""swirlc_b200 subpackage mirroring the reference module of the same name."""
