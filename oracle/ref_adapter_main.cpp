// ADAPTER DRIVER — TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own LeMonADE adapter, GPUScBFM_AB_Type<Ingredients>
// (src/pscbfm/GPUScBFM_AB_Type.h:22-197, compiled unchanged), over this engine: the class it wraps,
// UpdaterGPUScBFM_AB_Type, is include/bfm_updater.hpp (through oracle/ref_shim/adapter). LeMonADE is
// not installed, so the ingredients here are a minimal stand-in with the calls the adapter makes,
// and its base class and vector type come from tests/lemonade_stub. Built by oracle/Makefile
// (target `adapter`, output oracle/_ref/ref_adapter); run by the GPU tests against the oracle.
//
// Input (stdin): "box Lx Ly Lz", "periodic px py pz", "monomers n", n lines "x y z attribute", n
// lines "k id_1 .. id_k" (each monomer's neighbour list, in order), "run steps calls".
// Output (stdout): the positions after `calls` execute() calls of `steps` MCS each, one "x y z" line
// per monomer, then "age A".
#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "GPUScBFM_AB_Type.h"

namespace {

struct Monomer {
    int x = 0, y = 0, z = 0, tag = 1;
    int getX() const { return x; }
    int getY() const { return y; }
    int getZ() const { return z; }
    int getAttributeTag() const { return tag; }
    void setAllCoordinates(int a, int b, int c)
    {
        x = a;
        y = b;
        z = c;
    }
};

struct Molecules {
    std::vector<Monomer> m;
    std::vector<std::vector<int>> links;
    unsigned long long age = 0;
    std::size_t size() const { return m.size(); }
    Monomer& operator[](std::size_t i) { return m[i]; }
    Monomer const& operator[](std::size_t i) const { return m[i]; }
    std::size_t getNumLinks(std::size_t i) const { return links[i].size(); }
    int getNeighborIdx(std::size_t i, std::size_t k) const { return links[i][k]; }
    unsigned long long getAge() const { return age; }
    void setAge(unsigned long long a) { age = a; }
};

// the standard 108-vector bond set: squared lengths 4, 5, 6, 9 and 10 within [-4, 3]^3
struct Bondset {
    bool isValid(VectorInt3 const& v) const
    {
        int const l = v.x * v.x + v.y * v.y + v.z * v.z;
        return l == 4 || l == 5 || l == 6 || l == 9 || l == 10;
    }
};

struct Ingredients {
    typedef Molecules molecules_type;
    Molecules mol;
    Bondset bonds;
    unsigned box[3] = {0, 0, 0};
    bool periodic[3] = {true, true, true};
    Molecules const& getMolecules() const { return mol; }
    Molecules& modifyMolecules() { return mol; }
    Bondset const& getBondset() const { return bonds; }
    unsigned getBoxX() const { return box[0]; }
    unsigned getBoxY() const { return box[1]; }
    unsigned getBoxZ() const { return box[2]; }
    bool isPeriodicX() const { return periodic[0]; }
    bool isPeriodicY() const { return periodic[1]; }
    bool isPeriodicZ() const { return periodic[2]; }
};

bool expect(std::string const& word)
{
    std::string w;
    return (std::cin >> w) && w == word;
}

}  // namespace

int main()
{
    Ingredients ing;
    std::size_t n = 0;
    int px = 1, py = 1, pz = 1;
    if (!expect("box") || !(std::cin >> ing.box[0] >> ing.box[1] >> ing.box[2])) return 2;
    if (!expect("periodic") || !(std::cin >> px >> py >> pz)) return 2;
    ing.periodic[0] = px != 0;
    ing.periodic[1] = py != 0;
    ing.periodic[2] = pz != 0;
    if (!expect("monomers") || !(std::cin >> n)) return 2;
    ing.mol.m.resize(n);
    ing.mol.links.resize(n);
    for (std::size_t i = 0; i < n; ++i)
        if (!(std::cin >> ing.mol.m[i].x >> ing.mol.m[i].y >> ing.mol.m[i].z >> ing.mol.m[i].tag)) return 2;
    for (std::size_t i = 0; i < n; ++i) {
        std::size_t k = 0;
        if (!(std::cin >> k)) return 2;
        ing.mol.links[i].resize(k);
        for (std::size_t j = 0; j < k; ++j)
            if (!(std::cin >> ing.mol.links[i][j])) return 2;
    }
    uint32_t steps = 0, calls = 0;
    if (!expect("run") || !(std::cin >> steps >> calls)) return 2;
    try {
        GPUScBFM_AB_Type<Ingredients> updater(ing, steps, 0);
        updater.initialize();
        for (uint32_t c = 0; c < calls; ++c) updater.execute();
        for (auto const& q : ing.mol.m) std::printf("%d %d %d\n", q.x, q.y, q.z);
        std::printf("age %llu\n", ing.mol.getAge());
        updater.cleanup();
    } catch (std::exception const& e) {
        std::printf("error: %s\n", e.what());
        return 1;
    }
    return 0;
}
