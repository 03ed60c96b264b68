// A LeMonADE-style program (ingredients with the calls the reference adapter makes) driving the
// engine through include/bfm_lemonade.hpp; compiled by tests/test_capi.py and run by
// tests/test_gpu_api.py. Prints the final positions and the molecules' age.
#include "bfm_lemonade.hpp"
#include <cstdio>
#include <vector>
struct Monomer {
    int x = 0, y = 0, z = 0, tag = 1;
    int getX() const { return x; } int getY() const { return y; } int getZ() const { return z; }
    int getAttributeTag() const { return tag; }
    void setAllCoordinates(int a, int b, int c) { x = a; y = b; z = c; }
};
struct Molecules {
    std::vector<Monomer> m; std::vector<std::vector<int>> links; unsigned long long age = 0;
    std::size_t size() const { return m.size(); }
    Monomer& operator[](std::size_t i) { return m[i]; }
    Monomer const& operator[](std::size_t i) const { return m[i]; }
    std::size_t getNumLinks(std::size_t i) const { return links[i].size(); }
    int getNeighborIdx(std::size_t i, std::size_t k) const { return links[i][k]; }
    unsigned long long getAge() const { return age; } void setAge(unsigned long long a) { age = a; }
};
// the 108-vector set: squared lengths 4, 5, 6, 9 and 10 (all sign / permutations of (2,0,0), (2,1,0),
// (2,1,1), (2,2,1), (3,0,0), (3,1,0))
struct Bondset {
    bool isValid(VectorInt3 const& v) const
    {
        int const l = v.x * v.x + v.y * v.y + v.z * v.z;
        return l == 4 || l == 5 || l == 6 || l == 9 || l == 10;
    }
};
struct Ingredients {
    typedef Molecules molecules_type;
    Molecules mol; Bondset bonds;
    Molecules const& getMolecules() const { return mol; } Molecules& modifyMolecules() { return mol; }
    Bondset const& getBondset() const { return bonds; }
    unsigned getBoxX() const { return 32; } unsigned getBoxY() const { return 32; } unsigned getBoxZ() const { return 32; }
    bool isPeriodicX() const { return true; } bool isPeriodicY() const { return true; } bool isPeriodicZ() const { return true; }
};
int main() {
    Ingredients ing;
    ing.mol.m.resize(2); ing.mol.m[1].x = 2; ing.mol.links = {{1}, {0}};
    try {
        UpdaterB200ScBFM<Ingredients> gpu(ing, 100, 0);
        gpu.setSeed(7);
        gpu.initialize();
        gpu.execute();
        for (auto const& q : ing.mol.m) std::printf("%d %d %d\n", q.x, q.y, q.z);
        std::printf("age %llu\n", ing.mol.getAge());
        gpu.cleanup();
    } catch (std::exception const& e) { std::printf("error: %s\n", e.what()); return 1; }
    return 0;
}
