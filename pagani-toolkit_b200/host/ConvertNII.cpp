// ConvertNII.cpp -- nodal values (.nm) back to NIfTI volumes, as the
// reference's ConvertNII (U/ConvertNII/ConvertNII/ConvertNII.cpp:16-179):
//   ConvertNII <dir_with_nm_files> <mask.nii> [mask_threshold, default 0.5]
// Every *.nm in the directory holding N values, N being the number of mask
// voxels at or above the threshold, becomes <stem>.nii: a float32 volume with
// the mask's header whose mask voxels, in file order, take the N values and
// whose other voxels are zero.  A file whose N differs is reported, noted in
// BNA_time_log in the working directory, and skipped.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "formats.h"

int main(int argc, char** argv)
{
    if (argc < 3 || argc > 4) {
        fprintf(stderr,
                "Input format: ConvertNII Directory_containing_files_to_be_converted niiFile_for_mask "
                "[ |threshold_for_mask]\nFor example: ConvertNII X_dir mask.nii [ |0.4]\n");
        return 1;
    }
    pgio::Nifti mask;
    std::string err;
    if (!pgio::read_nifti(argv[2], mask, err)) {
        fprintf(stderr, "%s\n", err.c_str());
        return 1;
    }
    const double cut = argc == 4 ? atof(argv[3]) : 0.5;
    const long long V = (long long)mask.dims[0] * mask.dims[1] * mask.dims[2];
    long long nv = 0;
    for (long long k = 0; k < V; k++) nv += mask.data[k] >= (float)cut;
    std::vector<std::string> files = pgio::list_dir(argv[1], ".nm");
    printf("%zu files to be processed.\n", files.size());
    std::vector<float> vol((size_t)V);
    for (const std::string& fn : files) {
        const std::string path = pgio::join(argv[1], fn);
        printf("\nconvert analysis for %s ...\n", path.c_str());
        std::vector<float> x;
        if (!pgio::read_nm(path, x)) {
            printf("Can't open\t%s\n", path.c_str());
            continue;
        }
        if ((long long)x.size() != nv) {
            printf("Mask file doesn't match to the file %s\nContinue to convert the next file\n", fn.c_str());
            if (FILE* log = fopen("BNA_time_log", "a")) {
                fprintf(log, "Mask file doesn't match to the file %s\n", fn.c_str());
                fclose(log);
            }
            continue;
        }
        size_t l = 0;
        for (long long k = 0; k < V; k++) vol[(size_t)k] = mask.data[k] >= (float)cut ? x[l++] : 0.0f;
        if (!pgio::write_nifti_like(pgio::stem(path) + ".nii", mask, vol)) {
            fprintf(stderr, "cannot write %s.nii\n", pgio::stem(path).c_str());
            return 1;
        }
        printf("Convert to .nii completed!\n");
    }
    return 0;
}
