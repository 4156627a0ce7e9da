"""CPU oracle of the reference's hot path. TEST INFRASTRUCTURE ONLY: imported by
the tests, the smoke check and the benchmark's CPU-baseline leg, never by the
product package."""
