// Test-infrastructure shim (oracle only): the three-component integer
// vector that qes::Domain's (Vector3Int, Vector3Float) constructor reads.
#pragma once
class Vector3Int {
public:
  Vector3Int(int a = 0, int b = 0, int c = 0) : v{a, b, c} {}
  int &operator[](int i) { return v[i]; }
  const int &operator[](int i) const { return v[i]; }
private:
  int v[3];
};
