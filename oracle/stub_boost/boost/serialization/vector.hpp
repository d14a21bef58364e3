// Builder-written no-op stand-in: serialization is out of scope for the oracle.
#pragma once
#include <vector>
