// TEST INFRASTRUCTURE: a no-op stand-in for the HDF5Kit library so that the reference's
// hot-path sources compile without HDF5.  The reference only uses it in the attribute
// exporters (operator<< on hdf5::Group / hdf5::Dataset in Species.h, BField.h, EField.h,
// PartSpecies.h, ParamSet.h); nothing here writes anything.
#pragma once

#include <initializer_list>

namespace hdf5 {
struct Type {
};
struct Space {
    static Space scalar() { return {}; }
    template <class... A>
    static Space simple(A &&...) { return {}; }
    static Space simple(std::initializer_list<unsigned long>) { return {}; }
};
struct Attribute {
    template <class... A>
    Attribute &write(A &&...) { return *this; }
};
template <class T = void, class... A>
Type make_type(A &&...) { return {}; }
struct Group {
    template <class... A>
    Attribute attribute(A &&...) { return {}; }
};
struct Dataset {
    template <class... A>
    Attribute attribute(A &&...) { return {}; }
};
} // namespace hdf5
