// Small autotuner: times candidate launch configurations once per key and
// remembers the fastest for the rest of the process.
#pragma once

#include <functional>
#include <map>
#include <mutex>
#include <string>
#include <vector>

namespace ctb {

class Autotuner {
   public:
    static Autotuner& instance() {
        static Autotuner a;
        return a;
    }
    // Returns the cached choice for key, or times every candidate with
    // time_ms(candidate) (negative = candidate unusable) and caches the best.
    int pick(const std::string& key, const std::vector<int>& candidates,
             const std::function<double(int)>& time_ms, std::vector<double>* timings = nullptr) {
        {
            std::lock_guard<std::mutex> lk(mtx_);
            auto it = cache_.find(key);
            if (it != cache_.end()) return it->second;
        }
        int best = candidates.empty() ? 0 : candidates[0];
        double best_ms = -1;
        std::vector<double> t;
        for (int c : candidates) {
            const double ms = time_ms(c);
            t.push_back(ms);
            if (ms >= 0 && (best_ms < 0 || ms < best_ms)) {
                best_ms = ms;
                best = c;
            }
        }
        if (timings) *timings = t;
        std::lock_guard<std::mutex> lk(mtx_);
        cache_[key] = best;
        return best;
    }

   private:
    std::mutex mtx_;
    std::map<std::string, int> cache_;
};

}  // namespace ctb
