"""The test oracle (TEST INFRASTRUCTURE, not part of the product): see oracle.oracle."""
