// vlbm_run.cpp -- the reference program's host loop (src/CUDA/main.cu:47-606)
// on libvlbm's C ABI: the same YAML in (pyvisc's configuration file), the same
// files out (PATH/ID/ID_<var><step>.bin, ID_info.txt, ID_avgUz<step>.csv,
// ID_pCenters/pNodes<step>.csv, the checkpoint).
//
//   vlbm_run -c conf.yaml        (pyvisc's --conf-path, pyvisc/args_handler.py:24-30)
//
// Per step, as main.cu:270-507 with aux = step - INI_STEP:
//   save       = MACR_SAVE   && aux != 0 && aux % MACR_SAVE == 0
//   rep        = DATA_REPORT && aux != 0 && aux % DATA_REPORT == 0
//   checkpoint = CHECKPOINT_SAVE && aux != 0 && aux % CHECKPOINT_SAVE == 0
// The fluid kernel saves the macroscopics of the state it reads, before it
// collides (lbm.cu:247-261), so a save or report at iteration `step` holds the
// state after `step - INI_STEP` steps, and the final save, labelled with the
// loop's exit step, holds the state the last iteration read (main.cu:296,
// 524-527).  With spheres the macroscopics come from the IBM step that follows
// the fluid step (ibm.cu:544-648), i.e. after the iteration.  Particle files
// are written after the IBM step when step % IBM_PARTICLES_SAVE == 0
// (main.cu:391-393) and at the end (main.cu:532).  Checkpoints are written
// after the iteration (main.cu:452-458) and, when CHECKPOINT_SAVE is set, at
// the end (main.cu:547-548).  Steps between two such events run as one
// vlbm_step call.  MLUPS counts every node (main.cu:539-541) over wall-clock
// time including the saves, as the reference's timing window does.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>
#include "vlbm.h"

namespace {

int fail(const char* what, vlbm_status st) {
    std::fprintf(stderr, "vlbm_run: %s failed (status %d): %s\n", what, st, vlbm_last_error());
    return 1;
}

#define RUN(call)                                  \
    do {                                           \
        vlbm_status st_ = (call);                  \
        if (st_ != VLBM_OK) return fail(#call, st_); \
    } while (0)

bool every(int64_t interval, int64_t aux) { return interval > 0 && aux != 0 && aux % interval == 0; }

// Step field of getVarFilename (lbmReport.cpp:55-83), for the CSV the driver writes.
std::string step_field(uint32_t s) {
    std::string z;
    if (s == 0) {
        z = "000000";
    } else {
        uint32_t pot = 10;
        for (int k = 0; k < 12 && s * pot < 1000000u; ++k, pot *= 10) z.push_back('0');
    }
    return z + std::to_string(s);
}

// treatData + printTreatData (+ saveTreatData) of a report step (main.cu:468-485,
// treatData.cpp:462-496); returns the stop condition when DATA_STOP is set.
int report(vlbm_sim* sim, const vlbm_run_config& rc, int64_t step, std::vector<double>& avg_uz, bool* stop) {
    const int32_t ny = rc.cfg.ny;
    vlbm_treat t;
    RUN(vlbm_treat_data(sim, rc.resid_max, &t, avg_uz.data(), ny));
    std::printf("\n--------------------------------- TREATED DATA ---------------------------------\n");
    std::printf("                   Step: %lld\n", (long long)step);
    std::printf("               Residual: %.4e\n", t.residual);
    std::printf("           Avg. density: %.4e\n", t.avg_rho);
    std::printf("       Avg. Uz (y=NY/2): %.4e\n", avg_uz[ny / 2]);
    std::printf("--------------------------------------------------------------------------------\n");
    if (rc.data_save) {
        const std::string fn = std::string(rc.path_save) + "/" + rc.sim_id + "/" + rc.sim_id + "_avgUz" +
                               step_field((uint32_t)step) + ".csv";
        FILE* f = std::fopen(fn.c_str(), "w");
        if (!f) {
            std::printf("Error saving \"%s\" \nProbably wrong path!\n", fn.c_str());
        } else {
            std::fprintf(f, "y\tavg uz\n");
            for (int y = 0; y < ny; ++y) std::fprintf(f, "%d\t%.6e\n", y, avg_uz[y]);
            std::fclose(f);
        }
    }
    *stop = rc.data_stop && t.stop;
    if (*stop) std::printf("Stopping because of LBM\n");
    return 0;
}

}  // namespace

int main(int argc, char** argv) {
    const char* conf = nullptr;
    for (int k = 1; k < argc; ++k) {
        if ((!std::strcmp(argv[k], "-c") || !std::strcmp(argv[k], "--conf-path")) && k + 1 < argc) conf = argv[++k];
    }
    if (!conf) {
        std::fprintf(stderr, "usage: %s -c CONF.yaml\n", argv[0]);
        return 2;
    }
    vlbm_run_config rc;
    RUN(vlbm_run_config_load(conf, &rc, nullptr, 0));
    std::vector<vlbm_sphere> spheres(rc.n_spheres > 0 ? rc.n_spheres : 1);
    RUN(vlbm_run_config_load(conf, &rc, spheres.data(), rc.n_spheres));
    const char* path = rc.path_save;
    const char* id = rc.sim_id;
    const bool ibm = rc.use_ibm && rc.n_spheres > 0;

    vlbm_sim* sim = nullptr;
    RUN(vlbm_create(&rc.cfg, &sim));
    RUN(vlbm_set_builder(sim, rc.builder));
    if (ibm) RUN(vlbm_add_spheres(sim, &rc.ibm, spheres.data(), rc.n_spheres));
    // saveSimInfo before the loop (main.cu:169-170)
    RUN(vlbm_write_info(sim, path, id, 0, 0.0, (int32_t)rc.data_report, (int32_t)rc.macr_save, rc.u_max));

    int64_t step = rc.ini_step;
    if (rc.load_checkpoint) {   // loadSimCheckpoint (main.cu:199-202): continue from its step
        RUN(vlbm_load_checkpoint(sim, rc.load_folder, id));
        vlbm_info info;
        RUN(vlbm_get_info(sim, &info));
        step = info.step;
    }
    const int64_t first_step = step;
    std::vector<double> avg_uz(rc.cfg.ny);
    auto t0 = std::chrono::steady_clock::now();
    bool stopped = false;
    bool final_written = false;

    while (step < rc.steps) {
        const int64_t aux = step - rc.ini_step;
        const bool save = every(rc.macr_save, aux);
        const bool rep = every(rc.data_report, aux);
        const bool ckpt = every(rc.checkpoint_save, aux);
        const bool last = step + 1 >= rc.steps;
        if (!ibm) {
            // the macroscopics this iteration's fluid kernel saves: the state it reads
            if (save) RUN(vlbm_write_macr_bin(sim, path, id, (uint32_t)step, rc.export_forces));
            if (rep) {
                bool stop = false;
                if (report(sim, rc, step, avg_uz, &stop)) return 1;
                if (stop) {
                    stopped = true;
                    RUN(vlbm_write_macr_bin(sim, path, id, (uint32_t)step, rc.export_forces));
                    final_written = true;
                    break;
                }
            }
            if (last) {   // the final save holds what the last iteration read
                RUN(vlbm_write_macr_bin(sim, path, id, (uint32_t)rc.steps, rc.export_forces));
                final_written = true;
            }
        }
        // run up to the next iteration that has something to do
        int64_t n = 1;
        if (!save && !rep && !ckpt && !last) {
            int64_t next = rc.steps - 1;
            for (int64_t iv : {rc.macr_save, rc.data_report, rc.checkpoint_save}) {
                if (iv <= 0) continue;
                const int64_t a = aux + 1;
                const int64_t nxt = ((a + iv - 1) / iv) * iv + rc.ini_step;   // next multiple after aux
                if (nxt < next) next = nxt;
            }
            if (ibm && rc.particles_save > 0) {   // iteration nxt runs alone: its particle save follows it
                const int64_t nxt = ((step + rc.particles_save) / rc.particles_save) * rc.particles_save;
                if (nxt < next) next = nxt;
            }
            n = next > step ? next - step : 1;
        }
        if (ibm && rc.particles_save > 0 && step % rc.particles_save == 0) n = 1;
        RUN(vlbm_step(sim, (uint32_t)n));
        const int64_t done_step = step + n - 1;   // the iteration just completed
        step += n;
        if (ibm) {
            if (rc.particles_save > 0 && done_step % rc.particles_save == 0)
                RUN(vlbm_write_particles_csv(sim, path, id, (uint32_t)done_step, rc.particles_nodes_save));
            const int64_t a = done_step - rc.ini_step;
            if (every(rc.macr_save, a)) RUN(vlbm_write_macr_bin(sim, path, id, (uint32_t)done_step, rc.export_forces));
            if (every(rc.data_report, a)) {
                bool stop = false;
                if (report(sim, rc, done_step, avg_uz, &stop)) return 1;
                if (stop) {   // the reference leaves its loop before counting this iteration
                    stopped = true;
                    step = done_step;
                    break;
                }
            }
        }
        if (ckpt) RUN(vlbm_save_checkpoint(sim, path, id));
    }
    RUN(vlbm_sync(sim));
    const double elapsed = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    if (!final_written) RUN(vlbm_write_macr_bin(sim, path, id, (uint32_t)step, rc.export_forces));
    if (ibm) RUN(vlbm_write_particles_csv(sim, path, id, (uint32_t)step, rc.particles_nodes_save));
    if (rc.checkpoint_save != 0) RUN(vlbm_save_checkpoint(sim, path, id));
    const int64_t total = step - first_step;
    RUN(vlbm_write_info(sim, path, id, (uint64_t)total, elapsed, (int32_t)rc.data_report, (int32_t)rc.macr_save,
                        rc.u_max));
    const double nodes = (double)rc.cfg.nx * rc.cfg.ny * rc.cfg.nz;
    std::printf("\n              Steps: %lld%s\n", (long long)total, stopped ? " (stopped by the data condition)" : "");
    std::printf("              MLUPS: %f\n", elapsed > 0 ? total * nodes / 1e6 / elapsed : 0.0);
    std::printf("   Elapsed time (s): %f\n", elapsed);
    RUN(vlbm_destroy(sim));
    return 0;
}
