"""ORACLE -- test infrastructure only (CPU restatement of the reference's
lvl1 gate-bootstrapping path).  Never imported by the engine."""
