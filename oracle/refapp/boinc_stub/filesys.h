// Empty stand-in for a BOINC library header the reference app includes but
// whose declarations its standalone Linux build does not use.  Test
// infrastructure only.
#pragma once
