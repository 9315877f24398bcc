"""ORACLE TEST INFRASTRUCTURE (CPU checker); see oracle/oracle.py.  Never imported by the
product package."""
