namespace zerork {
const char *git_commit_id = "oracle-build";
const char *git_commit_timestamp = "none";
const char *git_branch_name = "none";
}
