// Test infrastructure: serialization is never used by the single-rank
// oracle/_ref build; this header only declares what the reference names.
#ifndef GFREF_SHIM_BOOST_PROPERTY_TREE_PTREE_SERIALIZATION_HPP
#define GFREF_SHIM_BOOST_PROPERTY_TREE_PTREE_SERIALIZATION_HPP
namespace boost {
namespace serialization {
class access;
}
}  // namespace boost
#endif
