// Test-infrastructure shim (oracle only): float counterpart of Vector3Int.
#pragma once
class Vector3Float {
public:
  Vector3Float(float a = 0, float b = 0, float c = 0) : v{a, b, c} {}
  float &operator[](int i) { return v[i]; }
  const float &operator[](int i) const { return v[i]; }
private:
  float v[3];
};
