// Test-infrastructure shim (oracle only): Wall.cpp includes the input-data
// header but the solver-coefficient routines never dereference it.
#pragma once
class WINDSInputData {};
