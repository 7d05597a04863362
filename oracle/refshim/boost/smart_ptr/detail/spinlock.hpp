/* Stand-in for the one Boost type the reference's neighbour lists name
 * (pvetex.h:6-12, kgraph.h:12-18).  The reference never runs two threads
 * (its OpenMP pragmas are commented out), so the lock does nothing; it only
 * has to be copyable so that std::vector<NNList> can resize. */
#ifndef NNM_REFSHIM_SPINLOCK_HPP
#define NNM_REFSHIM_SPINLOCK_HPP
namespace boost { namespace detail {
struct spinlock {
    int v_ = 0;
    void lock() {}
    bool try_lock() { return true; }
    void unlock() {}
};
}}
#endif
