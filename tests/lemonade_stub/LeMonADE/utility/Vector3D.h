// Test stand-in for LeMonADE's integer 3-vector (only the constructor the adapter uses).
#pragma once

struct VectorInt3 {
    int x, y, z;
    VectorInt3(int a, int b, int c) : x(a), y(b), z(c) {}
};
