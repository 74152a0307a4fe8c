"""TEST INFRASTRUCTURE: CPU checkers for the spiffe_b200 parity tests.

Only tests/, the smoke check and the benchmark's CPU-baseline leg import this
package, and only as a checker.  The product library never loads it.
"""
